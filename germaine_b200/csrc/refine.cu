// K6: FP64 residual r = b - M x of the 9-point operator for every
// right-hand side of every frequency, with per-(frequency, right-hand side)
// partial sums of |r|^2 and |b|^2, and the precision conversions of the
// mixed-precision refinement loop.  HBM-bound: per row 9 operator values
// (amortised over the right-hand sides) and x, b, r for each right-hand side.
#include "kernels.cuh"
#include "cplx.cuh"

namespace gm {

// Residual tile: RROWS consecutive unknowns of one matrix x RLANES
// right-hand sides, one warp per row at a time (the branch on the stencil's
// grid edges is warp-uniform, the 32 lanes read 32 consecutive right-hand
// sides of each neighbour row: one 512-byte load per neighbour), RGRP warps
// over the tile's rows.  The tile's operator values (9 per row, shared by
// every right-hand side) are staged in shared memory once.
constexpr int RROWS = 64;   // measured on 841 x 227: 32-row tiles took 15 % longer
constexpr int RLANES = 32;
constexpr int RGRP = 8;

// row tiles of the residual kernel for n unknowns (partial-sum blocks)
int residual_blocks(int n) { return (n + RROWS - 1) / RROWS; }

// Operator value M'[k][k+off(q)] for the selected orientation (M' = M or M^T,
// M = A^T in GM_OP_REF, M = A in GM_OP_EXACT); A[k][k+off(q)] = A9[q][k].
__device__ __forceinline__ double2 op_coef(const double2 *A9, int n, int nx, bool use_row, int q, int k) {
    if (use_row) return A9[(size_t)q * n + k];
    const int c = k + (q % 3 - 1) + (q / 3 - 1) * nx;
    return A9[(size_t)(8 - q) * n + c];
}

// out = b - M'x (PRODUCT = false) or out = M'x (PRODUCT = true), x of type
// InC, with per-(matrix, right-hand side) partial sums of |out|^2 and |b|^2
// into part[blockIdx.x][blockIdx.z][r][2].  OutC = double2 writes FP64;
// OutC = float2 writes the refinement right-hand side directly in the
// working precision of the substitution; WRITE = false forms the norms only.
template <class InC, class OutC, bool WRITE, bool PRODUCT>
__global__ void __launch_bounds__(RLANES *RGRP, 3) k_residual(ResidArgs a, const InC *__restrict__ xin, OutC *out,
                                                            double *part) {
    __shared__ double2 cf[9][RROWS];
    __shared__ unsigned short nbm[RROWS];   // per row: bit q set when neighbour q lies inside the grid
    __shared__ double red[2][RGRP][RLANES];
    const int fz = blockIdx.z;
    const int f = a.fmap ? a.fmap[fz] : fz;
    const int k0 = blockIdx.x * RROWS;
    const int r = blockIdx.y * RLANES + threadIdx.x;
    const bool use_row = (a.op_mode == GM_OP_EXACT) != (a.trans != 0);
    const double2 *A9 = a.A + (size_t)f * 9 * a.n;
    const int tid = threadIdx.y * RLANES + threadIdx.x;
    if (tid < RROWS) {   // the grid-edge tests once per row, not per right-hand side
        const int k = k0 + tid;
        unsigned m = 0;
        if (k < a.n) {
            const int x = k % a.nx, y = k / a.nx;
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const int xx = x + q % 3 - 1, yy = y + q / 3 - 1;
                if (xx >= 0 && xx < a.nx && yy >= 0 && yy < a.ny) m |= 1u << q;
            }
        }
        nbm[tid] = (unsigned short)m;
    }
    __syncthreads();
    for (int t = tid; t < 9 * RROWS; t += RLANES * RGRP) {
        const int q = t / RROWS, i = t % RROWS;
        cf[q][i] = (nbm[i] >> q) & 1 ? op_coef(A9, a.n, a.nx, use_row, q, k0 + i) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double rr = 0.0, bb = 0.0;
    if (r < a.nrhs) {
        const size_t per = (size_t)a.n * a.ldr;
        const size_t base = (size_t)f * per + r;
        const InC *X = xin + (size_t)(a.xmap ? a.xmap[fz] : f) * per + r;
        OutC *O = out ? out + (size_t)(a.omap ? a.omap[fz] : f) * per + r : nullptr;
        const bool spikes = !PRODUCT && a.spike_k;
        const int ks = spikes ? a.spike_k[r] : -1;
        const double2 amp = spikes ? a.spike_amp[f] : make_double2(0.0, 0.0);
        // neighbour q of row k is row k + dq[q]: offsets in elements of x
        int dq[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) dq[q] = ((q % 3 - 1) + (q / 3 - 1) * a.nx) * a.ldr;
#pragma unroll 2
        for (int i = threadIdx.y; i < RROWS; i += RGRP) {
            const int k = k0 + i;
            if (k >= a.n) break;
            const unsigned m = nbm[i];
            double2 bv = make_double2(0.0, 0.0);
            if (!PRODUCT) bv = spikes ? (k == ks ? amp : bv) : a.b[base + (size_t)k * a.ldr];
            double2 acc = bv;
            const InC *Xk = X + (size_t)k * a.ldr;
#pragma unroll
            for (int q = 0; q < 9; ++q)
                if ((m >> q) & 1) cfms(acc, cf[q][i], cto_d(Xk[dq[q]]));
            if (PRODUCT) acc = make_double2(-acc.x, -acc.y);
            if (WRITE) O[(size_t)k * a.ldr] = cconv<OutC>(acc);
            rr += acc.x * acc.x + acc.y * acc.y;
            bb += bv.x * bv.x + bv.y * bv.y;
        }
    }
    red[0][threadIdx.y][threadIdx.x] = rr;
    red[1][threadIdx.y][threadIdx.x] = bb;
    __syncthreads();
    if (threadIdx.y == 0 && r < a.nrhs) {
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int g = 0; g < RGRP; ++g) {
            s0 += red[0][g][threadIdx.x];
            s1 += red[1][g][threadIdx.x];
        }
        double *p = part + (((size_t)blockIdx.x * gridDim.z + fz) * a.nrhs + r) * 2;
        p[0] = s0;
        p[1] = s1;
    }
}

static int resid_nfz(const ResidArgs &a) { return a.fmap ? a.nfz : a.nf; }

template <class InC, class OutC, bool WRITE, bool PRODUCT>
static int launch_k6(const ResidArgs &a, const void *x, void *out, double *part, int max_blocks, cudaStream_t st) {
    const int nblk = residual_blocks(a.n);
    const int nfz = resid_nfz(a);
    if (nblk > max_blocks) return -1;
    if (nfz <= 0) return nblk;
    dim3 grid(nblk, (a.nrhs + RLANES - 1) / RLANES, nfz);
    (k_residual<InC, OutC, WRITE, PRODUCT><<<grid, dim3(RLANES, RGRP), 0, st>>>(
         a, reinterpret_cast<const InC *>(x), reinterpret_cast<OutC *>(out), part),
     note_launch());
    return nblk;
}

int launch_residual(const ResidArgs &a, double *part, int max_blocks, cudaStream_t st) {
    return launch_k6<double2, double2, true, false>(a, a.x, a.r, part, max_blocks, st);
}

template <class R>
int launch_residual_t(const ResidArgs &a, void *t, double *part, int max_blocks, cudaStream_t st) {
    if (t) return launch_k6<double2, cplx<R>, true, false>(a, a.x, t, part, max_blocks, st);
    return launch_k6<double2, cplx<R>, false, false>(a, a.x, nullptr, part, max_blocks, st);
}

template int launch_residual_t<double>(const ResidArgs &, void *, double *, int, cudaStream_t);
template int launch_residual_t<float>(const ResidArgs &, void *, double *, int, cudaStream_t);

template <class R>
int launch_matvec(const ResidArgs &a, const void *x, double2 *out, double *part, int max_blocks, cudaStream_t st) {
    return launch_k6<cplx<R>, double2, true, true>(a, x, out, part, max_blocks, st);
}

template int launch_matvec<double>(const ResidArgs &, const void *, double2 *, double *, int, cudaStream_t);
template int launch_matvec<float>(const ResidArgs &, const void *, double2 *, double *, int, cudaStream_t);

// out[c] = sum over blocks of part[blk][c]: 32 columns per CTA, eight
// warps over the blocks, then a fixed-order sum (deterministic)
__global__ void __launch_bounds__(256) k_reduce_norms(const double *part, int nblk, int cnt, double *out) {
    __shared__ double red[8][32];
    const int c = blockIdx.x * 32 + threadIdx.x;
    double s = 0.0;
    if (c < cnt)
        for (int b = threadIdx.y; b < nblk; b += 8) s += part[(size_t)b * cnt + c];
    red[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < cnt) {
        double t = 0.0;
#pragma unroll
        for (int g = 0; g < 8; ++g) t += red[g][threadIdx.x];
        out[c] = t;
    }
}

void launch_reduce_norms(const double *part, int nblk, int cnt, double *out, cudaStream_t st) {
    if (cnt <= 0) return;
    (k_reduce_norms<<<(cnt + 31) / 32, dim3(32, 8), 0, st>>>(part, nblk, cnt, out), note_launch());
}

template <class R>
__global__ void k_convert_down(const double2 *__restrict__ src, cplx<R> *__restrict__ dst, size_t count) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) dst[i] = cconv<cplx<R>>(src[i]);
}

template <class R>
__global__ void k_add_up(double2 *__restrict__ x, const cplx<R> *__restrict__ d, size_t count) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        const double2 v = cto_d(d[i]);
        double2 u = x[i];
        u.x += v.x;
        u.y += v.y;
        x[i] = u;
    }
}

template <class R>
void launch_convert_down(const double2 *src, void *dst, size_t count, cudaStream_t st) {
    if (!count) return;
    (k_convert_down<R><<<(unsigned)((count + 255) / 256), 256, 0, st>>>(src, reinterpret_cast<cplx<R> *>(dst), count), note_launch());
}

template <class R>
void launch_add_up(double2 *x, const void *d, size_t count, cudaStream_t st) {
    if (!count) return;
    (k_add_up<R><<<(unsigned)((count + 255) / 256), 256, 0, st>>>(x, reinterpret_cast<const cplx<R> *>(d), count), note_launch());
}

// x[f] += d[f] over the matrices f = fmap[0 .. nfz) (per_f entries each)
template <class R>
__global__ void k_add_up_f(double2 *__restrict__ x, const cplx<R> *__restrict__ d, size_t per_f, const int *fmap) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= per_f) return;
    const size_t o = (size_t)fmap[blockIdx.y] * per_f + i;
    const double2 v = cto_d(d[o]);
    double2 u = x[o];
    u.x += v.x;
    u.y += v.y;
    x[o] = u;
}

template <class R>
void launch_add_up_f(double2 *x, const void *d, size_t per_f, const int *fmap, int nfz, cudaStream_t st) {
    if (!per_f || nfz <= 0) return;
    dim3 grid((unsigned)((per_f + 255) / 256), nfz);
    (k_add_up_f<R><<<grid, 256, 0, st>>>(x, reinterpret_cast<const cplx<R> *>(d), per_f, fmap), note_launch());
}

template void launch_add_up_f<double>(double2 *, const void *, size_t, const int *, int, cudaStream_t);
template void launch_add_up_f<float>(double2 *, const void *, size_t, const int *, int, cudaStream_t);

// Loads the residual / conversion kernels (see preload_solve_kernels).
void preload_refine_kernels() {
    cudaFuncAttributes fa;
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, double2, true, false>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, double2, false, false>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, float2, true, false>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, float2, false, false>);
    cudaFuncGetAttributes(&fa, (const void *)k_reduce_norms);
    cudaFuncGetAttributes(&fa, (const void *)k_convert_down<double>);
    cudaFuncGetAttributes(&fa, (const void *)k_convert_down<float>);
    cudaFuncGetAttributes(&fa, (const void *)k_add_up<double>);
    cudaFuncGetAttributes(&fa, (const void *)k_add_up<float>);
}

template void launch_convert_down<double>(const double2 *, void *, size_t, cudaStream_t);
template void launch_convert_down<float>(const double2 *, void *, size_t, cudaStream_t);
template void launch_add_up<double>(double2 *, const void *, size_t, cudaStream_t);
template void launch_add_up<float>(double2 *, const void *, size_t, cudaStream_t);

}  // namespace gm
