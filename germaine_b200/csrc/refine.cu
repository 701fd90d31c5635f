// K6: FP64 residual r = b - M x of the 9-point operator for every
// right-hand side of every frequency, with per-(frequency, right-hand side)
// partial sums of |r|^2 and |b|^2, and the precision conversions of the
// mixed-precision refinement loop.  HBM-bound: per row 9 operator values
// (amortised over the right-hand sides) and x, b, r for each right-hand side.
#include "kernels.cuh"
#include "cplx.cuh"

namespace gm {

constexpr int RROWS = 64;  // rows per CTA of the residual kernel

// Operator value M'[k][k+off(q)] for the selected orientation (M' = M or M^T,
// M = A^T in GM_OP_REF, M = A in GM_OP_EXACT); A[k][k+off(q)] = A9[q][k].
__device__ __forceinline__ double2 op_coef(const double2 *A9, int n, int nx, bool use_row, int q, int k) {
    if (use_row) return A9[(size_t)q * n + k];
    const int c = k + (q % 3 - 1) + (q / 3 - 1) * nx;
    return A9[(size_t)(8 - q) * n + c];
}

// OutC = double2 writes r = b - M'x; OutC = cplx<R> writes the refinement
// right-hand side directly in the working precision of the substitution.
// WRITE = false computes only the norms (a check that is expected to pass).
template <class OutC, bool WRITE = true>
__global__ void __launch_bounds__(128) k_residual(ResidArgs a, OutC *out, double *part) {
    const int f = blockIdx.y;
    const int k0 = blockIdx.x * RROWS, k1 = min(a.n, k0 + RROWS);
    const bool use_row = (a.op_mode == GM_OP_EXACT) != (a.trans != 0);
    const double2 *A9 = a.A + (size_t)f * 9 * a.n;
    const size_t base = (size_t)f * a.n * a.ldr;
    const double2 amp = a.spike_k ? a.spike_amp[f] : make_double2(0.0, 0.0);
    for (int r = threadIdx.x; r < a.nrhs; r += blockDim.x) {
        double rr = 0.0, bb = 0.0;
        const int ks = a.spike_k ? a.spike_k[r] : -1;
        for (int k = k0; k < k1; ++k) {
            const int x = k % a.nx, y = k / a.nx;
            const double2 bv = a.spike_k ? (k == ks ? amp : make_double2(0.0, 0.0)) : a.b[base + (size_t)k * a.ldr + r];
            double2 acc = bv;
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const int xx = x + q % 3 - 1, yy = y + q / 3 - 1;
                if (xx < 0 || xx >= a.nx || yy < 0 || yy >= a.ny) continue;
                const double2 m = op_coef(A9, a.n, a.nx, use_row, q, k);
                const double2 xv = a.x[base + (size_t)(yy * a.nx + xx) * a.ldr + r];
                cfms(acc, m, xv);
            }
            if (WRITE) out[base + (size_t)k * a.ldr + r] = cconv<OutC>(acc);
            rr += acc.x * acc.x + acc.y * acc.y;
            bb += bv.x * bv.x + bv.y * bv.y;
        }
        double *p = part + (((size_t)blockIdx.x * gridDim.y + f) * a.nrhs + r) * 2;
        p[0] = rr;
        p[1] = bb;
    }
}

int launch_residual(const ResidArgs &a, double *part, int max_blocks, cudaStream_t st) {
    const int nblk = (a.n + RROWS - 1) / RROWS;
    if (nblk > max_blocks) return -1;
    (k_residual<double2><<<dim3(nblk, a.nf), 128, 0, st>>>(a, a.r, part), note_launch());
    return nblk;
}

template <class R>
int launch_residual_t(const ResidArgs &a, void *t, double *part, int max_blocks, cudaStream_t st) {
    const int nblk = (a.n + RROWS - 1) / RROWS;
    if (nblk > max_blocks) return -1;
    if (t) (k_residual<cplx<R>, true><<<dim3(nblk, a.nf), 128, 0, st>>>(a, reinterpret_cast<cplx<R> *>(t), part), note_launch());
    else (k_residual<cplx<R>, false><<<dim3(nblk, a.nf), 128, 0, st>>>(a, nullptr, part), note_launch());
    return nblk;
}

template int launch_residual_t<double>(const ResidArgs &, void *, double *, int, cudaStream_t);
template int launch_residual_t<float>(const ResidArgs &, void *, double *, int, cudaStream_t);

// out[c] = sum over blocks of part[blk][c] (fixed order: deterministic)
__global__ void k_reduce_norms(const double *part, int nblk, int cnt, double *out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cnt) return;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[(size_t)b * cnt + c];
    out[c] = s;
}

void launch_reduce_norms(const double *part, int nblk, int cnt, double *out, cudaStream_t st) {
    (k_reduce_norms<<<(cnt + 255) / 256, 256, 0, st>>>(part, nblk, cnt, out), note_launch());
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

template void launch_convert_down<double>(const double2 *, void *, size_t, cudaStream_t);
template void launch_convert_down<float>(const double2 *, void *, size_t, cudaStream_t);
template void launch_add_up<double>(double2 *, const void *, size_t, cudaStream_t);
template void launch_add_up<float>(double2 *, const void *, size_t, cudaStream_t);

}  // namespace gm
