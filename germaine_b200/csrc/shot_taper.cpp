// Host drop-ins for the reference's per-shot gradient tapers, for callers
// that form per-shot gradients themselves (the engine applies the same
// tapers inside its gradient stack, gm_set_shot_taper):
//   gm_taper_grad_shot   taper_grad_shot  (src/taper_grad_shot.c:11)
//   gm_taper_grad_shot1  taper_grad_shot1 (src/taper_grad_shot1.c:11)
// Float results identical to the reference's (host_setup.c evaluates the
// coefficients in the reference's float / double order); the radial taper
// touches only the points within reach of a centre, where the reference
// multiplies the whole grid by 1.0f elsewhere, and the squares are clipped
// to the grid where the reference writes past its arrays.
#include "common.hpp"
#include "germaine_gpu.h"
#include "host_setup.h"

extern "C" int gm_taper_grad_shot(int nx, int ny, float dh, float srtradius, int nshots, const float *src_x,
                                  const float *src_y, int ntr, const int32_t *rec_x, const int32_t *rec_y, int ishot,
                                  float *grad) {
    if (nx <= 0 || ny <= 0 || !(dh > 0.0f) || !(srtradius > 0.0f) || !grad || nshots <= 0 || !src_x || !src_y ||
        ntr < 0 || (ntr > 0 && (!rec_x || !rec_y)))
        return gm::fail(GM_ERROR_INVALID, "gm_taper_grad_shot: bad argument");
    if (ishot < 0 || ishot >= nshots)
        return gm::fail(GM_ERROR_INVALID, "gm_taper_grad_shot: shot %d of %d", ishot, nshots);
    gmh_taper_grad_shot(nx, ny, dh, srtradius, src_x, src_y, ntr, rec_x, rec_y, ishot, grad);
    return GM_OK;
}

extern "C" int gm_taper_grad_shot1(int nx, int ny, float dh, int filtsize, int nshots, const float *src_x,
                                   const float *src_y, int ntr, const int32_t *rec_x, const int32_t *rec_y,
                                   float *grad) {
    if (nx <= 0 || ny <= 0 || !(dh > 0.0f) || filtsize < 0 || !grad || nshots < 0 ||
        (nshots > 0 && (!src_x || !src_y)) || ntr < 0 || (ntr > 0 && (!rec_x || !rec_y)))
        return gm::fail(GM_ERROR_INVALID, "gm_taper_grad_shot1: bad argument");
    gmh_taper_grad_shot1(nx, ny, dh, filtsize, nshots, src_x, src_y, ntr, rec_x, rec_y, grad, nullptr);
    return GM_OK;
}
