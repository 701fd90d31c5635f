// K6b: the vector kernels of GMRES-IR, the refinement used for matrices
// whose plain refinement contracts slowly (low frequency or strong PML
// contrast under complex64 factors).  GMRES runs on the correction equation
// M' d = r in FP64 with the working-precision factors as a right
// preconditioner (flexible form: the preconditioned vectors z_j are kept),
// so the Arnoldi relation M' Z = V H holds to FP64 rounding and the
// correction is exact to that level; its cost is one substitution and one
// FP64 operator product per iteration, like a refinement sweep.
//
// Vectors are [slot][n][nrhs] (right-hand side fastest), one slot per matrix
// of the GMRES set; every kernel runs over the launch's list of slots
// (zmap) and treats each right-hand side as its own column: a GMRES run per
// (matrix, right-hand side).  The Krylov vectors V_i are kept unnormalised
// (their norms beta_i live on the host), so no separate scaling pass is
// needed: every coefficient below already carries the 1 / beta_i.
// Reductions give per-(row block, column) partial sums that a fixed-order
// block reduction (k_reduce_norms) finishes: deterministic results.
#include "kernels.cuh"
#include "cplx.cuh"

namespace gm {

constexpr int GLANES = 32;   // right-hand sides per CTA (lanes)
constexpr int GGRP = 8;      // warps per CTA, over rows
constexpr int GROWS = 256;   // rows per CTA

// Z[zs] = (R)(V[zs] * s[j][r]) for launch position j, slot zs = zmap[j]
template <class R>
__global__ void __launch_bounds__(256) k_scale_down(const double2 *__restrict__ V, cplx<R> *__restrict__ Z,
                                                    const double *__restrict__ s, const int *zmap, int n, int nrhs) {
    const size_t per = (size_t)n * nrhs;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= per) return;
    const size_t o = (size_t)zmap[blockIdx.y] * per + i;
    const double c = s[(size_t)blockIdx.y * nrhs + i % nrhs];
    const double2 v = V[o];
    Z[o] = cconv<cplx<R>>(make_double2(v.x * c, v.y * c));
}

// part[blk][j][r][i] = sum over the block's rows of conj(V_i[k][r]) W[k][r],
// i < nv (and i = nv: |W[k][r]|^2 in the real part)
template <int MAXV>
__global__ void __launch_bounds__(GLANES *GGRP) k_dots(const double2 *__restrict__ V, size_t vstride, int nv,
                                                      const double2 *__restrict__ W, const int *zmap, int n,
                                                      int nrhs, double *part) {
    __shared__ double red[GGRP][GLANES][2];
    const int j = blockIdx.z;
    const int r = blockIdx.y * GLANES + threadIdx.x;
    const size_t per = (size_t)n * nrhs;
    const size_t base = (size_t)zmap[j] * per + r;
    double2 acc[MAXV + 1];
#pragma unroll
    for (int i = 0; i <= MAXV; ++i) acc[i] = make_double2(0.0, 0.0);
    if (r < nrhs) {
        const int k0 = blockIdx.x * GROWS, k1 = min(n, k0 + GROWS);
        for (int k = k0 + threadIdx.y; k < k1; k += GGRP) {
            const size_t o = base + (size_t)k * nrhs;
            const double2 w = W[o];
#pragma unroll
            for (int i = 0; i < MAXV; ++i) {
                if (i >= nv) break;
                const double2 v = V[(size_t)i * vstride + o];
                acc[i].x = fma(v.x, w.x, fma(v.y, w.y, acc[i].x));   // conj(v) * w
                acc[i].y = fma(v.x, w.y, fma(-v.y, w.x, acc[i].y));
            }
            acc[MAXV].x = fma(w.x, w.x, fma(w.y, w.y, acc[MAXV].x));
        }
    }
    const int ncoef = nv + 1;
    for (int i = 0; i < ncoef; ++i) {
        double2 a = make_double2(0.0, 0.0);
#pragma unroll
        for (int q = 0; q <= MAXV; ++q)
            if (q == (i < nv ? i : MAXV)) a = acc[q];
        red[threadIdx.y][threadIdx.x][0] = a.x;
        red[threadIdx.y][threadIdx.x][1] = a.y;
        __syncthreads();
        if (threadIdx.y == 0 && r < nrhs) {
            double sx = 0.0, sy = 0.0;
#pragma unroll
            for (int g = 0; g < GGRP; ++g) {
                sx += red[g][threadIdx.x][0];
                sy += red[g][threadIdx.x][1];
            }
            double *p = part + ((((size_t)blockIdx.x * gridDim.z + j) * nrhs + r) * ncoef + i) * 2;
            p[0] = sx;
            p[1] = sy;
        }
        __syncthreads();
    }
}

// W[k][r] -= sum_{i < nv} coef[j][r][i] V_i[k][r]; part[blk][j][r] = the
// block's sum of the updated |W[k][r]|^2
template <int MAXV>
__global__ void __launch_bounds__(GLANES *GGRP) k_gs_update(const double2 *__restrict__ V, size_t vstride, int nv,
                                                           double2 *__restrict__ W, const double2 *__restrict__ coef,
                                                           const int *zmap, int n, int nrhs, double *part) {
    __shared__ double red[GGRP][GLANES];
    const int j = blockIdx.z;
    const int r = blockIdx.y * GLANES + threadIdx.x;
    const size_t per = (size_t)n * nrhs;
    const size_t base = (size_t)zmap[j] * per + r;
    double nrm = 0.0;
    if (r < nrhs) {
        double2 c[MAXV];
#pragma unroll
        for (int i = 0; i < MAXV; ++i)
            c[i] = i < nv ? coef[((size_t)j * nrhs + r) * MAXV + i] : make_double2(0.0, 0.0);
        const int k0 = blockIdx.x * GROWS, k1 = min(n, k0 + GROWS);
        for (int k = k0 + threadIdx.y; k < k1; k += GGRP) {
            const size_t o = base + (size_t)k * nrhs;
            double2 w = W[o];
#pragma unroll
            for (int i = 0; i < MAXV; ++i) {
                if (i >= nv) break;
                cfms(w, c[i], V[(size_t)i * vstride + o]);
            }
            W[o] = w;
            nrm = fma(w.x, w.x, fma(w.y, w.y, nrm));
        }
    }
    red[threadIdx.y][threadIdx.x] = nrm;
    __syncthreads();
    if (threadIdx.y == 0 && r < nrhs) {
        double s = 0.0;
#pragma unroll
        for (int g = 0; g < GGRP; ++g) s += red[g][threadIdx.x];
        part[((size_t)blockIdx.x * gridDim.z + j) * nrhs + r] = s;
    }
}

// x[fmap[j]][k][r] += sum_{i < nz} y[j][r][i] Z_i[zmap[j]][k][r]
template <class R, int MAXV>
__global__ void __launch_bounds__(256) k_x_update(double2 *__restrict__ x, const cplx<R> *__restrict__ Z,
                                                  size_t zstride, int nz, const double2 *__restrict__ y,
                                                  const int *fmap, const int *zmap, int n, int nrhs) {
    const size_t per = (size_t)n * nrhs;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= per) return;
    const int j = blockIdx.y, r = (int)(i % nrhs);
    const size_t oz = (size_t)zmap[j] * per + i;
    const size_t ox = (size_t)fmap[j] * per + i;
    double2 acc = x[ox];
#pragma unroll
    for (int q = 0; q < MAXV; ++q) {
        if (q >= nz) break;
        cfma(acc, y[((size_t)j * nrhs + r) * MAXV + q], cto_d(Z[(size_t)q * zstride + oz]));
    }
    x[ox] = acc;
}

static int gm_blocks(int n) { return (n + GROWS - 1) / GROWS; }

template <class R>
void launch_scale_down(const double2 *V, void *Z, const double *s, const int *zmap, int nj, int n, int nrhs,
                       cudaStream_t st) {
    const size_t per = (size_t)n * nrhs;
    if (!per || nj <= 0) return;
    dim3 grid((unsigned)((per + 255) / 256), nj);
    (k_scale_down<R><<<grid, 256, 0, st>>>(V, reinterpret_cast<cplx<R> *>(Z), s, zmap, n, nrhs), note_launch());
}

int launch_dots(const double2 *V, size_t vstride, int nv, const double2 *W, const int *zmap, int nj, int n, int nrhs,
                double *part, cudaStream_t st) {
    const int nblk = gm_blocks(n);
    if (nj <= 0) return nblk;
    dim3 grid(nblk, (nrhs + GLANES - 1) / GLANES, nj);
    (k_dots<kGmresStride><<<grid, dim3(GLANES, GGRP), 0, st>>>(V, vstride, nv, W, zmap, n, nrhs, part),
     note_launch());
    return nblk;
}

int launch_gs_update(const double2 *V, size_t vstride, int nv, double2 *W, const double2 *coef, const int *zmap,
                     int nj, int n, int nrhs, double *part, cudaStream_t st) {
    const int nblk = gm_blocks(n);
    if (nj <= 0) return nblk;
    dim3 grid(nblk, (nrhs + GLANES - 1) / GLANES, nj);
    (k_gs_update<kGmresStride><<<grid, dim3(GLANES, GGRP), 0, st>>>(V, vstride, nv, W, coef, zmap, n, nrhs,
                                                                             part),
     note_launch());
    return nblk;
}

template <class R>
void launch_x_update(double2 *x, const void *Z, size_t zstride, int nz, const double2 *y, const int *fmap,
                     const int *zmap, int nj, int n, int nrhs, cudaStream_t st) {
    const size_t per = (size_t)n * nrhs;
    if (!per || nj <= 0 || nz <= 0) return;
    dim3 grid((unsigned)((per + 255) / 256), nj);
    (k_x_update<R, kGmresStride><<<grid, 256, 0, st>>>(x, reinterpret_cast<const cplx<R> *>(Z), zstride, nz, y,
                                                           fmap, zmap, n, nrhs),
     note_launch());
}

template void launch_scale_down<double>(const double2 *, void *, const double *, const int *, int, int, int,
                                        cudaStream_t);
template void launch_scale_down<float>(const double2 *, void *, const double *, const int *, int, int, int,
                                       cudaStream_t);
template void launch_x_update<double>(double2 *, const void *, size_t, int, const double2 *, const int *,
                                      const int *, int, int, int, cudaStream_t);
template void launch_x_update<float>(double2 *, const void *, size_t, int, const double2 *, const int *,
                                     const int *, int, int, int, cudaStream_t);

void preload_gmres_kernels() {
    cudaFuncAttributes fa;
    cudaFuncGetAttributes(&fa, (const void *)k_scale_down<double>);
    cudaFuncGetAttributes(&fa, (const void *)k_scale_down<float>);
    cudaFuncGetAttributes(&fa, (const void *)k_dots<kGmresStride>);
    cudaFuncGetAttributes(&fa, (const void *)k_gs_update<kGmresStride>);
    cudaFuncGetAttributes(&fa, (const void *)k_x_update<double, kGmresStride>);
    cudaFuncGetAttributes(&fa, (const void *)k_x_update<float, kGmresStride>);
}

}  // namespace gm
