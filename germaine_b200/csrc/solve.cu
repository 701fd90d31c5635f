// K5: multi-right-hand-side forward/backward substitution through the
// multifrontal factors (the replacement of one umfpack_zi_solve call per
// shot, src/AC/forward_shot_AC.c:88, by one block solve over every shot of
// every frequency).
//
// Right-hand sides / solutions are [nf][n][ldr] complex, right-hand side
// fastest.  One CTA (8 warps) owns one (front, frequency, slice of up to 32
// right-hand sides); lane l of every warp works on right-hand side l, so all
// vector traffic is a coalesced row of the slice.
//   forward (leaves -> root): gather the front vector (own rows of x plus
//     the children's update vectors, by the same inverse maps as the
//     extend-add), then for each 32-pivot block: triangular solve of the
//     block -- one warp per right-hand side, lane p holding unknown p, the
//     eliminated value broadcast by warp shuffle (no block barrier inside
//     the block) -- and a rank-32 update of the rows below from 64-row tiles
//     of L staged in shared memory; y goes back to x at the pivots, the
//     trailing rows stay in the front-vector workspace as this front's update
//     for its parent;
//   backward (root -> leaves): t = y - U12 x2 (x2 = final values of the
//     ancestors' variables), then blocked back substitution with U11.
// trans = 1 solves M^T x = b with the same factors: M^T = U^T L^T, so the
// forward pass runs with U^T (non-unit diagonal) and the backward pass with
// L^T (unit diagonal); only the indexing of the factor changes.
#include "kernels.cuh"
#include "cplx.cuh"

namespace gm {

constexpr int SNB = 32;    // pivot block
constexpr int RT = 64;     // row tile of the updates
constexpr int NWARP = 8;

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

__device__ __forceinline__ double2 shfl(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ float2 shfl(float2 v, int src) {
    return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

template <class C>
struct SolveSmem {
    C D[SNB][SNB + 1];   // diagonal block of the current pivot block
    C Y[SNB][SNB + 1];   // solved block [pivot][rhs], or a ring block of x
    C L[RT][SNB + 1];    // factor tile [row][pivot]
};

// Stage the factor tile T[row][q] = (lower ? L' : U')(i0 + row, c0 + q),
// row < rows, q < qb, coalesced along the factor's contiguous index.
template <class C, bool TRANS>
__device__ __forceinline__ void stage_tile(C (*T)[SNB + 1], const C *F, int f, int i0, int rows, int c0, int qb) {
    if (!TRANS) {   // column-major: contiguous along the row index
        for (int t = threadIdx.x; t < RT * SNB; t += blockDim.x) {
            const int row = t % RT, q = t / RT;
            if (row < rows && q < qb) T[row][q] = F[(i0 + row) + (size_t)(c0 + q) * f];
        }
    } else {        // transposed access: contiguous along the pivot index
        for (int t = threadIdx.x; t < RT * SNB; t += blockDim.x) {
            const int q = t % SNB, row = t / SNB;
            if (row < rows && q < qb) T[row][q] = F[(c0 + q) + (size_t)(i0 + row) * f];
        }
    }
}

// V[i0 + row][lane] -= sum_q T[row][q] * Y[q][lane] over the staged tile;
// warp w owns rows w + 8j.
template <class C>
__device__ __forceinline__ void tile_update(const C (*T)[SNB + 1], const C (*Y)[SNB + 1], int qb, C *V, int ldr,
                                            int i0, int rows, int rn) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    C acc[RT / NWARP];
#pragma unroll
    for (int j = 0; j < RT / NWARP; ++j) acc[j] = czero<C>();
    for (int q = 0; q < qb; ++q) {
        const C y = Y[q][lane];
#pragma unroll
        for (int j = 0; j < RT / NWARP; ++j) cfma(acc[j], T[warp + NWARP * j][q], y);
    }
    if (lane < rn) {
#pragma unroll
        for (int j = 0; j < RT / NWARP; ++j) {
            const int row = warp + NWARP * j;
            if (row < rows) {
                C &d = V[(size_t)(i0 + row) * ldr + lane];
                d = csub(d, acc[j]);
            }
        }
    }
}

template <class R, bool TRANS>
__global__ void __launch_bounds__(256) k_fwd(SolveArgs<R> a, int lvl_first) {
    using C = cplx<R>;
    extern __shared__ unsigned char smem_raw[];
    SolveSmem<C> &sm = *reinterpret_cast<SolveSmem<C> *>(smem_raw);
    const int node = a.s.lvl_nodes[lvl_first + blockIdx.y];
    const int f = a.s.nfront[node], s = a.s.npiv[node];
    const int r0 = blockIdx.x * a.rch;
    const int rn = min(a.rch, a.nrhs - r0);
    if (rn <= 0) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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

    // gather the front vector (warp per row, lane per right-hand side)
    for (int i = warp; i < f; i += NWARP) {
        if (lane < rn) {
            C v = i < s ? X[(size_t)vars[i] * a.ldr + lane] : czero<C>();
            if (W0) { const int q = inv[i]; if (q >= 0) v = cadd(v, W0[(size_t)q * a.ldr + lane]); }
            if (W1) { const int q = inv[f + i]; if (q >= 0) v = cadd(v, W1[(size_t)q * a.ldr + lane]); }
            W[(size_t)i * a.ldr + lane] = v;
        }
    }

    for (int k0 = 0; k0 < s; k0 += SNB) {
        const int kb = min(SNB, s - k0);
        if (!TRANS) {
            for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
                const int p = t % kb, q = t / kb;
                if (p >= q) sm.D[p][q] = F[(k0 + p) + (size_t)(k0 + q) * f];
            }
        } else {
            for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
                const int q = t % kb, p = t / kb;
                if (p >= q) sm.D[p][q] = F[(k0 + q) + (size_t)(k0 + p) * f];
            }
        }
        __syncthreads();   // D staged; W rows of this block final
        for (int r = warp; r < rn; r += NWARP) {
            C y = lane < kb ? W[(size_t)(k0 + lane) * a.ldr + r] : czero<C>();
            for (int p = 0; p < kb; ++p) {
                if (TRANS && lane == p) y = cmul(y, crcp(sm.D[p][p]));
                const C yp = shfl(y, p);
                if (lane > p && lane < kb) cfms(y, sm.D[lane][p], yp);
            }
            if (lane < kb) sm.Y[lane][r] = y;
        }
        __syncthreads();
        for (int q = warp; q < kb; q += NWARP) {
            if (lane < rn) {
                const C y = sm.Y[q][lane];
                W[(size_t)(k0 + q) * a.ldr + lane] = y;
                X[(size_t)vars[k0 + q] * a.ldr + lane] = y;
            }
        }
        for (int i0 = k0 + kb; i0 < f; i0 += RT) {
            const int rows = min(RT, f - i0);
            stage_tile<C, TRANS>(sm.L, F, f, i0, rows, k0, kb);
            __syncthreads();
            tile_update<C>(sm.L, sm.Y, kb, W, a.ldr, i0, rows, rn);
            __syncthreads();
        }
    }
}

template <class R, bool TRANS>
__global__ void __launch_bounds__(256) k_bwd(SolveArgs<R> a, int lvl_first) {
    using C = cplx<R>;
    extern __shared__ unsigned char smem_raw[];
    SolveSmem<C> &sm = *reinterpret_cast<SolveSmem<C> *>(smem_raw);
    const int node = a.s.lvl_nodes[lvl_first + blockIdx.y];
    const int f = a.s.nfront[node], s = a.s.npiv[node];
    const int r0 = blockIdx.x * a.rch;
    const int rn = min(a.rch, a.nrhs - r0);
    if (rn <= 0) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t fz = blockIdx.z;
    const C *F = reinterpret_cast<const C *>(a.front) + fz * a.s.front_total + a.s.front_off[node];
    C *X = reinterpret_cast<C *>(a.x) + fz * (size_t)a.s.n * a.ldr + r0;
    C *T = reinterpret_cast<C *>(a.w) + fz * (size_t)a.s.rhs_total * a.ldr + r0 +
           (size_t)a.s.rhs_off[node] * a.ldr;   // rows 0..s-1 hold y from the forward pass
    const int *vars = a.s.vars + a.s.var_off[node];

    // t = y - U'12 x2: 64-row tiles of t, ring in blocks of 32
    for (int i0 = 0; i0 < s; i0 += RT) {
        const int rows = min(RT, s - i0);
        for (int j0 = s; j0 < f; j0 += SNB) {
            const int jb = min(SNB, f - j0);
            for (int q = warp; q < jb; q += NWARP)
                sm.Y[q][lane] = lane < rn ? X[(size_t)vars[j0 + q] * a.ldr + lane] : czero<C>();
            stage_tile<C, TRANS>(sm.L, F, f, i0, rows, j0, jb);
            __syncthreads();
            tile_update<C>(sm.L, sm.Y, jb, T, a.ldr, i0, rows, rn);
            __syncthreads();
        }
    }
    // blocked back substitution with U'11, last block first
    const int nblk = (s + SNB - 1) / SNB;
    for (int b = nblk - 1; b >= 0; --b) {
        const int k0 = b * SNB, kb = min(SNB, s - k0);
        if (!TRANS) {
            for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
                const int p = t % kb, q = t / kb;
                if (p <= q) sm.D[p][q] = F[(k0 + p) + (size_t)(k0 + q) * f];
            }
        } else {
            for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
                const int q = t % kb, p = t / kb;
                if (p <= q) sm.D[p][q] = F[(k0 + q) + (size_t)(k0 + p) * f];
            }
        }
        __syncthreads();
        for (int r = warp; r < rn; r += NWARP) {
            C t = lane < kb ? T[(size_t)(k0 + lane) * a.ldr + r] : czero<C>();
            for (int p = kb - 1; p >= 0; --p) {
                if (!TRANS && lane == p) t = cmul(t, crcp(sm.D[p][p]));
                const C xp = shfl(t, p);
                if (lane < p) cfms(t, sm.D[lane][p], xp);
            }
            if (lane < kb) sm.Y[lane][r] = t;
        }
        __syncthreads();
        for (int q = warp; q < kb; q += NWARP)
            if (lane < rn) X[(size_t)vars[k0 + q] * a.ldr + lane] = sm.Y[q][lane];
        for (int i0 = 0; i0 < k0; i0 += RT) {
            const int rows = min(RT, k0 - i0);
            stage_tile<C, TRANS>(sm.L, F, f, i0, rows, k0, kb);
            __syncthreads();
            tile_update<C>(sm.L, sm.Y, kb, T, a.ldr, i0, rows, rn);
            __syncthreads();
        }
    }
}

template <class R>
static void set_smem(const void *fn) {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SolveSmem<cplx<R>>));
}

template <class R>
void launch_solve_forward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    if (L.count == 0) return;
    static bool attr = false;
    if (!attr) {
        set_smem<R>((const void *)k_fwd<R, false>);
        set_smem<R>((const void *)k_fwd<R, true>);
        attr = true;
    }
    const size_t smem = sizeof(SolveSmem<cplx<R>>);
    dim3 grid((a.nrhs + a.rch - 1) / a.rch, L.count, a.nf);
    if (a.trans) (k_fwd<R, true><<<grid, 32 * NWARP, smem, st>>>(a, L.first), note_launch());
    else (k_fwd<R, false><<<grid, 32 * NWARP, smem, st>>>(a, L.first), note_launch());
}

template <class R>
void launch_solve_backward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    if (L.count == 0) return;
    static bool attr = false;
    if (!attr) {
        set_smem<R>((const void *)k_bwd<R, false>);
        set_smem<R>((const void *)k_bwd<R, true>);
        attr = true;
    }
    const size_t smem = sizeof(SolveSmem<cplx<R>>);
    dim3 grid((a.nrhs + a.rch - 1) / a.rch, L.count, a.nf);
    if (a.trans) (k_bwd<R, true><<<grid, 32 * NWARP, smem, st>>>(a, L.first), note_launch());
    else (k_bwd<R, false><<<grid, 32 * NWARP, smem, st>>>(a, L.first), note_launch());
}

template void launch_solve_forward_level<double>(const SolveArgs<double> &, const LevelInfo &, cudaStream_t);
template void launch_solve_forward_level<float>(const SolveArgs<float> &, const LevelInfo &, cudaStream_t);
template void launch_solve_backward_level<double>(const SolveArgs<double> &, const LevelInfo &, cudaStream_t);
template void launch_solve_backward_level<float>(const SolveArgs<float> &, const LevelInfo &, cudaStream_t);

}  // namespace gm
