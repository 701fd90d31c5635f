// Launch wrappers of the per-shot epilogue kernels (epilogue.cu).
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace gm {

struct GradArgs {
    int n, nf, ns, te;
    const double2 *xf, *xa;     // forward / adjoint solutions [nf][n][ns]
    const double2 *stfu;        // w/|w| per (f, s)
    const double2 *om2, *om;    // per frequency
    const float *m0, *m1;       // vp, rho (AC)
    const float *frame;         // PML taper coefficient per grid point
    const unsigned char *passes;
    double *g0, *g1;            // [n] outputs (FP64)
    // per-shot taper (0 none; 1 radial around the shot's source and every
    // receiver; 2 the term replaced by 1e-5 on the marked squares)
    int nx, shot_taper;
    const double *taper_rec;    // [n] product of the receivers' radial coefficients (1)
    const int4 *taper_win;      // per shot: first column, first row (0-based), width, height of its source window (1)
    const int *taper_off;       // per shot: offset of its window's coefficients in taper_src (1)
    const float *taper_src;     // source-window coefficients, row-major per window (1)
    const unsigned char *taper_mask;   // [n] 1 on the squares (2)
};

struct HessArgs {
    int n, nf, te;
    const double *sqf, *sqg;    // [nf][n] sums of |F|^2 over shots, |G|^2 over receivers (sqg NULL: shin)
    const double *w0, *w1;      // per frequency |coefficient|^2 of J (AC: |2 Omega^2|^2; TE: |Omega|^2, |Omega^2|^2)
    const float *m0, *m1;       // vp, rho (AC)
    const float *frame;
    const unsigned char *passes;
    double *h0, *h1;            // [n] outputs (FP64)
    float *f0, *f1;             // [n] float outputs: the sum rounded to float, then tapered in float
};

void launch_spikes(double2 *b, int n, int nf, int ns, const int *ksrc, const double2 *amp, cudaStream_t st);
void launch_gather_seis(const double2 *x, int n, int nf, int ns, int ntr, const int *krec, float2 *seis, double2 *cal,
                        cudaStream_t st);
void launch_field(const double2 *x, int n, int nf, int ns, float2 *field, cudaStream_t st);
void launch_residual_shot(const double2 *cal, const float2 *obs, int nfs, int ntr, int stf_inv, int misfit,
                          int invmat, int zeroing, double2 *res, double *l2, double2 *stf, cudaStream_t st);
void launch_adjoint_src(double2 *b, int n, int nf, int ns, int ntr, const int *kadj, const double2 *res, double dh2,
                        cudaStream_t st);
void launch_gradient(const GradArgs &a, cudaStream_t st);
// exact discrete AC gradient of GM_OP_EXACT (w: mass weights a, b, c)
void launch_gradient_exact(const GradArgs &a, const float w[3], cudaStream_t st);
void launch_hess_sq(const double2 *x, int n, int nf, int ns, double *sq, int accumulate, cudaStream_t st);
void launch_hess_final(const HessArgs &a, cudaStream_t st);

}  // namespace gm
