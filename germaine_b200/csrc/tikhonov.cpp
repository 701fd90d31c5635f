// Host drop-ins for the TE inversion's Tikhonov regularisation, applied by
// the reference's FWI loop and line searches after grad_obj_TE / obj_TE:
//   gm_tikhonov_cost_te  Tikhonov_cost_TE (src/TE/Tikhonov_cost_TE.c:10)
//   gm_tikhonov_grad_te  Tikhonov_grad_TE (src/TE/Tikhonov_grad_TE.c:10)
// Float results identical to the reference's (host_setup.c keeps its
// float / double evaluation order).  Grids are row-major [NY][NX] with the
// PML frame, the gradients those gm_grad_obj returns for TE.
#include <vector>

#include "common.hpp"
#include "germaine_gpu.h"
#include "host_setup.h"

namespace {

int check_args(const char *who, int nx, int ny, int idx, int idy, float dh, float norm1, float norm2,
               const float *sigma, const float *epsilon) {
    if (nx <= 0 || ny <= 0 || idx <= 0 || idy <= 0 || !(dh > 0.0f) || norm1 == 0.0f || norm2 == 0.0f || !sigma ||
        !epsilon)
        return gm::fail(GM_ERROR_INVALID, "%s: bad argument", who);
    return GM_OK;
}

}  // namespace

extern "C" int gm_tikhonov_cost_te(int nx, int ny, int idx, int idy, float dh, float mat1_norm, float mat2_norm,
                                   float beta_mat1, float beta_mat2, float lambda_1, float lambda_2,
                                   const float *sigma, const float *epsilon, float l2, float *l2_out) {
    if (int rc = check_args("gm_tikhonov_cost_te", nx, ny, idx, idy, dh, mat1_norm, mat2_norm, sigma, epsilon))
        return rc;
    if (!l2_out) return gm::fail(GM_ERROR_INVALID, "gm_tikhonov_cost_te: no output");
    std::vector<float> work(2 * (size_t)nx * ny);
    *l2_out = gmh_tikhonov_cost_te(nx, ny, idx, idy, dh, mat1_norm, mat2_norm, beta_mat1, beta_mat2, lambda_1,
                                   lambda_2, sigma, epsilon, l2, work.data());
    return GM_OK;
}

extern "C" int gm_tikhonov_grad_te(int nx, int ny, int idx, int idy, float dh, float mat1_norm, float mat2_norm,
                                   float beta_mat1, float beta_mat2, float lambda_1, float lambda_2,
                                   const float *sigma, const float *epsilon, float *grad_sigma,
                                   float *grad_epsilon) {
    if (int rc = check_args("gm_tikhonov_grad_te", nx, ny, idx, idy, dh, mat1_norm, mat2_norm, sigma, epsilon))
        return rc;
    if (!grad_sigma || !grad_epsilon) return gm::fail(GM_ERROR_INVALID, "gm_tikhonov_grad_te: no gradient");
    std::vector<float> work(2 * (size_t)nx * ny);
    gmh_tikhonov_grad_te(nx, ny, idx, idy, dh, mat1_norm, mat2_norm, beta_mat1, beta_mat2, lambda_1, lambda_2, sigma,
                         epsilon, grad_sigma, grad_epsilon, work.data());
    return GM_OK;
}
