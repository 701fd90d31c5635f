// K5: multi-right-hand-side forward/backward substitution through the
// multifrontal factors (the replacement of one umfpack_zi_solve call per
// shot, src/AC/forward_shot_AC.c:88, by one block solve over every shot of
// every frequency).
//
// Right-hand sides / solutions are [nf][n][ldr] complex, right-hand side
// fastest, so a front gathers whole contiguous rows.  Each CTA owns one
// (front, frequency, RC-wide slice of right-hand sides):
//   forward (leaves -> root): gather the front vector (own rows of x plus the
//     children's update vectors, by the same inverse maps as the extend-add),
//     then blocked substitution with L (NB pivots at a time: triangular solve
//     of the block in shared memory, then a rank-NB update of the rows
//     below); y goes back to x at the pivots and the trailing rows stay in
//     the front-vector workspace as this front's update for its parent;
//   backward (root -> leaves): t = y - U12 x2 with x2 gathered from the
//     already final ancestors, then blocked back substitution with U11.
// trans = 1 solves M^T x = b with the same factors: M^T = U^T L^T, so the
// forward pass runs with U^T (non-unit diagonal) and the backward pass with
// L^T (unit diagonal) -- only the indexing of the factor changes.
#include "kernels.cuh"
#include "cplx.cuh"

namespace gm {

constexpr int SNB = 32;  // substitution block

template <class C, bool TRANS>
__device__ __forceinline__ C lower_el(const C *F, int f, int i, int c) {
    // forward-pass factor L'(i, c), i >= c
    return TRANS ? F[c + (size_t)i * f] : F[i + (size_t)c * f];
}
template <class C, bool TRANS>
__device__ __forceinline__ C upper_el(const C *F, int f, int i, int c) {
    // backward-pass factor U'(i, c), i <= c
    return TRANS ? F[c + (size_t)i * f] : F[i + (size_t)c * f];
}

template <class R, int RC, bool TRANS>
__global__ void __launch_bounds__(256) k_fwd(SolveArgs<R> a, int lvl_first) {
    using C = cplx<R>;
    const int node = a.s.lvl_nodes[lvl_first + blockIdx.y];
    const int f = a.s.nfront[node], s = a.s.npiv[node];
    const int r0 = blockIdx.x * RC;
    const int rn = min(RC, a.nrhs - r0);
    if (rn <= 0) return;
    const size_t fz = blockIdx.z;
    const C *F = reinterpret_cast<const C *>(a.front) + fz * a.s.front_total + a.s.front_off[node];
    C *X = reinterpret_cast<C *>(a.x) + fz * (size_t)a.s.n * a.ldr + r0;
    C *Wall = reinterpret_cast<C *>(a.w) + fz * (size_t)a.s.rhs_total * a.ldr + r0;
    C *W = Wall + (size_t)a.s.rhs_off[node] * a.ldr;
    const int *vars = a.s.vars + a.s.var_off[node];
    const int *inv = a.s.inv + a.s.inv_off[node];
    const int c0 = a.s.child0[node], c1 = a.s.child1[node];
    const C *W0 = c0 >= 0 ? Wall + (size_t)(a.s.rhs_off[c0] + a.s.npiv[c0]) * a.ldr : nullptr;
    const C *W1 = c1 >= 0 ? Wall + (size_t)(a.s.rhs_off[c1] + a.s.npiv[c1]) * a.ldr : nullptr;

    // gather the front vector
    for (int t = threadIdx.x; t < f * RC; t += blockDim.x) {
        const int i = t / RC, r = t % RC;
        if (r >= rn) continue;
        C v = i < s ? X[(size_t)vars[i] * a.ldr + r] : czero<C>();
        if (W0) { const int q = inv[i]; if (q >= 0) v = cadd(v, W0[(size_t)q * a.ldr + r]); }
        if (W1) { const int q = inv[f + i]; if (q >= 0) v = cadd(v, W1[(size_t)q * a.ldr + r]); }
        W[(size_t)i * a.ldr + r] = v;
    }
    __syncthreads();

    __shared__ C Ys[SNB][RC];
    __shared__ C Ds[SNB][SNB + 1];
    for (int k0 = 0; k0 < s; k0 += SNB) {
        const int kb = min(SNB, s - k0);
        for (int t = threadIdx.x; t < SNB * RC; t += blockDim.x) {
            const int q = t / RC, r = t % RC;
            Ys[q][r] = (q < kb && r < rn) ? W[(size_t)(k0 + q) * a.ldr + r] : czero<C>();
        }
        for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
            const int i = t % kb, c = t / kb;
            Ds[i][c] = i >= c ? lower_el<C, TRANS>(F, f, k0 + i, k0 + c) : czero<C>();
        }
        __syncthreads();
        for (int p = 0; p < kb; ++p) {
            if (TRANS) {
                if (threadIdx.x < RC) Ys[p][threadIdx.x] = cmul(Ys[p][threadIdx.x], crcp(Ds[p][p]));
                __syncthreads();
            }
            for (int t = threadIdx.x; t < (kb - p - 1) * RC; t += blockDim.x) {
                const int q = p + 1 + t / RC, r = t % RC;
                cfms(Ys[q][r], Ds[q][p], Ys[p][r]);
            }
            __syncthreads();
        }
        for (int t = threadIdx.x; t < kb * RC; t += blockDim.x) {
            const int q = t / RC, r = t % RC;
            if (r < rn) {
                W[(size_t)(k0 + q) * a.ldr + r] = Ys[q][r];
                X[(size_t)vars[k0 + q] * a.ldr + r] = Ys[q][r];
            }
        }
        // rows below the block: W[i] -= L'(i, k0:k0+kb) * Y
        for (int i = k0 + kb + threadIdx.x; i < f; i += blockDim.x) {
            C acc[RC];
#pragma unroll
            for (int r = 0; r < RC; ++r) acc[r] = czero<C>();
            for (int q = 0; q < kb; ++q) {
                const C l = lower_el<C, TRANS>(F, f, i, k0 + q);
#pragma unroll
                for (int r = 0; r < RC; ++r) cfma(acc[r], l, Ys[q][r]);
            }
            C *wr = W + (size_t)i * a.ldr;
#pragma unroll
            for (int r = 0; r < RC; ++r)
                if (r < rn) wr[r] = csub(wr[r], acc[r]);
        }
        __syncthreads();
    }
}

template <class R, int RC, bool TRANS>
__global__ void __launch_bounds__(256) k_bwd(SolveArgs<R> a, int lvl_first) {
    using C = cplx<R>;
    const int node = a.s.lvl_nodes[lvl_first + blockIdx.y];
    const int f = a.s.nfront[node], s = a.s.npiv[node];
    const int r0 = blockIdx.x * RC;
    const int rn = min(RC, a.nrhs - r0);
    if (rn <= 0) return;
    const size_t fz = blockIdx.z;
    const C *F = reinterpret_cast<const C *>(a.front) + fz * a.s.front_total + a.s.front_off[node];
    C *X = reinterpret_cast<C *>(a.x) + fz * (size_t)a.s.n * a.ldr + r0;
    C *T = reinterpret_cast<C *>(a.w) + fz * (size_t)a.s.rhs_total * a.ldr + r0 +
           (size_t)a.s.rhs_off[node] * a.ldr;   // rows 0..s-1 hold y from the forward pass
    const int *vars = a.s.vars + a.s.var_off[node];

    __shared__ C Ys[SNB][RC];
    __shared__ C Ds[SNB][SNB + 1];
    // t = y - U'12 x2, ring blocks of SNB at a time
    for (int j0 = s; j0 < f; j0 += SNB) {
        const int jb = min(SNB, f - j0);
        for (int t = threadIdx.x; t < SNB * RC; t += blockDim.x) {
            const int q = t / RC, r = t % RC;
            Ys[q][r] = (q < jb && r < rn) ? X[(size_t)vars[j0 + q] * a.ldr + r] : czero<C>();
        }
        __syncthreads();
        for (int i = threadIdx.x; i < s; i += blockDim.x) {
            C acc[RC];
#pragma unroll
            for (int r = 0; r < RC; ++r) acc[r] = czero<C>();
            for (int q = 0; q < jb; ++q) {
                const C u = upper_el<C, TRANS>(F, f, i, j0 + q);
#pragma unroll
                for (int r = 0; r < RC; ++r) cfma(acc[r], u, Ys[q][r]);
            }
            C *tr = T + (size_t)i * a.ldr;
#pragma unroll
            for (int r = 0; r < RC; ++r)
                if (r < rn) tr[r] = csub(tr[r], acc[r]);
        }
        __syncthreads();
    }
    // blocked back substitution with U'11, last block first
    const int nblk = (s + SNB - 1) / SNB;
    for (int b = nblk - 1; b >= 0; --b) {
        const int k0 = b * SNB, kb = min(SNB, s - k0);
        for (int t = threadIdx.x; t < SNB * RC; t += blockDim.x) {
            const int q = t / RC, r = t % RC;
            Ys[q][r] = (q < kb && r < rn) ? T[(size_t)(k0 + q) * a.ldr + r] : czero<C>();
        }
        for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
            const int i = t % kb, c = t / kb;
            Ds[i][c] = i <= c ? upper_el<C, TRANS>(F, f, k0 + i, k0 + c) : czero<C>();
        }
        __syncthreads();
        for (int p = kb - 1; p >= 0; --p) {
            if (!TRANS) {
                if (threadIdx.x < RC) Ys[p][threadIdx.x] = cmul(Ys[p][threadIdx.x], crcp(Ds[p][p]));
                __syncthreads();
            }
            for (int t = threadIdx.x; t < p * RC; t += blockDim.x) {
                const int q = t / RC, r = t % RC;
                cfms(Ys[q][r], Ds[q][p], Ys[p][r]);
            }
            __syncthreads();
        }
        for (int t = threadIdx.x; t < kb * RC; t += blockDim.x) {
            const int q = t / RC, r = t % RC;
            if (r < rn) X[(size_t)vars[k0 + q] * a.ldr + r] = Ys[q][r];
        }
        // rows above the block: T[i] -= U'(i, k0:k0+kb) * x_blk
        for (int i = threadIdx.x; i < k0; i += blockDim.x) {
            C acc[RC];
#pragma unroll
            for (int r = 0; r < RC; ++r) acc[r] = czero<C>();
            for (int q = 0; q < kb; ++q) {
                const C u = upper_el<C, TRANS>(F, f, i, k0 + q);
#pragma unroll
                for (int r = 0; r < RC; ++r) cfma(acc[r], u, Ys[q][r]);
            }
            C *tr = T + (size_t)i * a.ldr;
#pragma unroll
            for (int r = 0; r < RC; ++r)
                if (r < rn) tr[r] = csub(tr[r], acc[r]);
        }
        __syncthreads();
    }
}

template <class R> struct SolveRC;
template <> struct SolveRC<double> { static constexpr int v = 8; };
template <> struct SolveRC<float> { static constexpr int v = 16; };

template <class R>
void launch_solve_forward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    constexpr int RC = SolveRC<R>::v;
    if (L.count == 0) return;
    dim3 grid((a.nrhs + RC - 1) / RC, L.count, a.nf);
    if (a.trans) k_fwd<R, RC, true><<<grid, 256, 0, st>>>(a, L.first);
    else k_fwd<R, RC, false><<<grid, 256, 0, st>>>(a, L.first);
}

template <class R>
void launch_solve_backward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    constexpr int RC = SolveRC<R>::v;
    if (L.count == 0) return;
    dim3 grid((a.nrhs + RC - 1) / RC, L.count, a.nf);
    if (a.trans) k_bwd<R, RC, true><<<grid, 256, 0, st>>>(a, L.first);
    else k_bwd<R, RC, false><<<grid, 256, 0, st>>>(a, L.first);
}

template void launch_solve_forward_level<double>(const SolveArgs<double> &, const LevelInfo &, cudaStream_t);
template void launch_solve_forward_level<float>(const SolveArgs<float> &, const LevelInfo &, cudaStream_t);
template void launch_solve_backward_level<double>(const SolveArgs<double> &, const LevelInfo &, cudaStream_t);
template void launch_solve_backward_level<float>(const SolveArgs<float> &, const LevelInfo &, cudaStream_t);

}  // namespace gm
