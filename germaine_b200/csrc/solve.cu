// K5: multi-right-hand-side forward/backward substitution through the
// multifrontal factors (the replacement of one umfpack_zi_solve call per
// shot, src/AC/forward_shot_AC.c:88, by one block solve over every shot of
// every frequency).
//
// Right-hand sides / solutions are [nf][n][ldr] complex, right-hand side
// fastest.  Work units are (front, frequency, slice of 32 or 40 right-hand
// sides).  The factorisation stores, in every 32 x 32 diagonal block, the
// inverses of the block's triangles, so every step below is a small GEMM on
// CUDA cores: 128 threads, each owning a (RT/16) x B complex register tile
// of an RT-row x 8B-right-hand-side output tile, operands staged in shared
// memory.
//
// Pivot rows are solved in place in x (their rows of x hold the right-hand
// side, then y, then the solution); the workspace w holds only each front's
// update vector for its parent (its ring rows).  Per elimination-tree level:
//   forward  (leaves -> root)
//     k_fwd_piv   add the children's update vectors (by the extend-add
//                 inverse maps) into x at the pivots, then per 32-pivot block:
//                 y_b = L_bb^-1 x_b, x_rest -= L_rb y_b over the remaining
//                 pivot rows;
//     k_fwd_ring  w_ring = (children's update vectors at the ring rows)
//                 - L_ring,piv * y over 64-row tiles of the ring (many CTAs
//                 per front: the wide part of the level);
//   backward (root -> leaves)
//     k_bwd_ring  x_piv -= U_piv,ring * x_ring (x_ring = final values of the
//                 ancestors' variables), 64-row tiles of the pivot rows;
//     k_bwd_piv   per block from the last: x_b = U_bb^-1 x_b,
//                 x_above -= U_ab x_b.
// trans = 1 solves M^T x = b with the same factors: M^T = U^T L^T, the
// forward pass runs with U^T and the backward pass with L^T; only the
// factor indexing and which stored inverse is used change.
#include <cstdlib>

#include "kernels.cuh"
#include "cplx.cuh"
#include "async_copy.cuh"

namespace gm {

constexpr int SNB = 32;   // pivot block (= factorisation block)
constexpr int NT = 128;   // threads per CTA
// Template parameters of the kernels:
//   RT (output rows per tile, 64 or 32): 64-row tiles reuse each staged
//      right-hand-side row over more factor rows; 32-row tiles halve the
//      accumulators and the factor tile, so more CTAs fit on an SM -- the
//      better trade on the small fronts of the lower tree levels;
//   B (right-hand sides per CTA = 8 B): every slice re-stages the front's
//      factor tiles, so wider slices read the factors fewer times.

// Tile rows are padded by SPAD elements: the complex128 tile product reads
// 8 x 4 fragments (4 pivots x 8 rows), which a stride of RT + 2 spreads over
// distinct shared-memory banks.
constexpr int SPAD = 2;

template <class C, int RT, int B>
struct SolveSmem {
    C L[SNB][RT + SPAD];       // factor tile, [pivot q][row]
    C Y[SNB][8 * B + SPAD];    // right operand, [pivot q][rhs]
};

// factor element M'(i, c) of the forward (L') or backward (U') factor:
// F[i + c f] for M x = b, F[c + i f] for M^T x = b
template <class C, bool TRANS>
__device__ __forceinline__ C elem(const C *F, int f, int i, int c) {
    return TRANS ? F[c + (size_t)i * f] : F[i + (size_t)c * f];
}

// The staging helpers below issue asynchronous copies (every load of the
// tile in flight at once, no register round trip); the tile is complete
// after staged_sync().
//
// sm.L[q][row] = M'(i0 + row, c0 + q) for row < rows, q < qb.  Entries
// outside are left as they are: tile_mma reads only q < qb, and rows >= rows
// (or right-hand sides >= rn) only feed accumulators that are never stored,
// so partial tiles stage only what they use.
// (the _p forms take the tile by pointer and the participating threads as
// lt = 0 .. nt - 1; the SolveSmem forms are the CTA-wide ones)
template <class C, bool TRANS, int RT>
__device__ __forceinline__ void stage_factor_p(C (*L)[RT + SPAD], const C *F, int f, int i0, int rows, int c0, int qb,
                                               int lt, int nt) {
    if (!TRANS) {
        for (int t = lt; t < RT * qb; t += nt) {
            const int row = t % RT, q = t / RT;
            if (row < rows) cp_async_elem(&L[q][row], F + (i0 + row) + (size_t)(c0 + q) * f);
        }
    } else {
        for (int t = lt; t < SNB * rows; t += nt) {
            const int q = t % SNB, row = t / SNB;
            if (q < qb) cp_async_elem(&L[q][row], F + (c0 + q) + (size_t)(i0 + row) * f);
        }
    }
}
template <class C, bool TRANS, int RT, int B>
__device__ __forceinline__ void stage_factor(SolveSmem<C, RT, B> &sm, const C *F, int f, int i0, int rows, int c0, int qb) {
    stage_factor_p<C, TRANS, RT>(sm.L, F, f, i0, rows, c0, qb, threadIdx.x, NT);
}

// sm.L[q][p] = the inverse diagonal-block operator of pivot block k0:
//   FWD && !TRANS: L^-1        FWD && TRANS: (U^-1)^T
//   !FWD && !TRANS: U^-1       !FWD && TRANS: (L^-1)^T
// The stored block holds L^-1 strictly below the diagonal (unit diagonal
// implied) and U^-1 on and above it.
template <class C, bool FWD, bool TRANS, int RT>
__device__ __forceinline__ void stage_dinv_p(C (*L)[RT + SPAD], const C *F, int f, int k0, int kb, int lt, int nt) {
    for (int t = lt; t < SNB * kb; t += nt) {
        const int p = t % SNB, q = t / SNB;   // operator entry (p, q) -> L[q][p], q < kb
        if (p >= kb) continue;
        const bool lower_src = FWD != TRANS;         // L^-1 (or its transpose) wanted
        const int r = TRANS ? q : p, c = TRANS ? p : q;  // position in the stored block
        const bool stored = lower_src ? r > c : r <= c;
        if (stored) {
            cp_async_elem(&L[q][p], F + (k0 + r) + (size_t)(k0 + c) * f);
        } else {
            using RR = decltype(L[0][0].x);
            L[q][p] = (lower_src && r == c) ? mk(RR(1), RR(0)) : czero<C>();
        }
    }
}
template <class C, bool FWD, bool TRANS, int RT, int B>
__device__ __forceinline__ void stage_dinv(SolveSmem<C, RT, B> &sm, const C *F, int f, int k0, int kb) {
    stage_dinv_p<C, FWD, TRANS, RT>(sm.L, F, f, k0, kb, threadIdx.x, NT);
}

// Per-thread accumulators of an RT x 8B complex output tile (128 threads,
// lt = 0 .. 127), in the layout of the tile product that fills them.
template <class C, int RT, int B>
struct TileAcc;

// complex64: CUDA-core FMAs; thread (tr, tc) = (lt / 8, lt % 8) owns rows
// tr + 16 i and columns tc + 8 j
template <int RT, int B>
struct TileAcc<float2, RT, B> {
    static constexpr int NR = RT / 16, NC = B;
    float2 v[NR][NC];
    __device__ __forceinline__ static int row(int i, int lt) { return lt / 8 + 16 * i; }
    __device__ __forceinline__ static int col(int j, int lt) { return lt % 8 + 8 * j; }
};

// complex128: FP64 matrix instructions (mma.sync m8n8k4 f64) on 8 x 8
// blocks; warp w owns row blocks w + 4 i, lane l row 8 (w + 4 i) + l / 4 of
// them and columns 8 c + 2 (l % 4) + {0, 1} of every column block c
template <int RT, int B>
struct TileAcc<double2, RT, B> {
    static constexpr int NR = RT / 32, NC = 2 * B;
    double2 v[NR][NC];
    __device__ __forceinline__ static int row(int i, int lt) { return 8 * ((lt >> 5) + 4 * i) + ((lt & 31) >> 2); }
    __device__ __forceinline__ static int col(int j, int lt) { return 8 * (j >> 1) + 2 * (lt & 3) + (j & 1); }
};

template <class C, int RT, int B>
__device__ __forceinline__ void zero_acc(TileAcc<C, RT, B> &acc) {
#pragma unroll
    for (int i = 0; i < TileAcc<C, RT, B>::NR; ++i)
#pragma unroll
        for (int j = 0; j < TileAcc<C, RT, B>::NC; ++j) acc.v[i][j] = czero<C>();
}

// f(row, col, value) for the thread's accumulators with row < rows, col < rn
template <class C, int RT, int B, class F>
__device__ __forceinline__ void for_acc(const TileAcc<C, RT, B> &acc, int rows, int rn, int lt, F f) {
    using A = TileAcc<C, RT, B>;
#pragma unroll
    for (int i = 0; i < A::NR; ++i) {
        const int row = A::row(i, lt);
        if (row >= rows) continue;
#pragma unroll
        for (int j = 0; j < A::NC; ++j) {
            const int col = A::col(j, lt);
            if (col < rn) f(row, col, acc.v[i][j]);
        }
    }
}

// acc += L'[rows x qb] Y[qb x rn]: L[q][row] holds operator entry (row, q),
// Y[q][col] the right operand.  Rows >= `rows` and columns >= rn of the
// tile only feed accumulators that are never stored; row and column groups
// that lie entirely outside are skipped warp-uniformly, so small fronts and
// short slices do not pay for the full tile.  TRI: 0 a full operator;
// TRI_LOWER / TRI_UPPER a triangular one (the diagonal-block inverses),
// whose column q has no entries above / below row q: row groups that column
// q does not reach are skipped for that q.
constexpr int TRI_LOWER = 1, TRI_UPPER = 2;

// complex64: each thread accumulates its 16-row-strided rows x 8-column-
// strided columns with CUDA-core FMAs, one pivot q at a time
template <int TRI, int RT, int B>
__device__ __forceinline__ void tile_mma_p(const float2 (*L)[RT + SPAD], const float2 (*Y)[8 * B + SPAD], int qb,
                                           TileAcc<float2, RT, B> &acc, int rows, int rn, int lt) {
    constexpr int A = RT / 16;
    const int tr = lt / 8, tc = lt % 8;
    const int wrow = (lt >> 5) * 4;   // a warp owns rows 4w .. 4w + 3 of each 16-row group
    const int na = rows <= wrow ? 0 : min(A, (rows - wrow + 15) / 16);
    const int nb = min(B, (rn + 7) / 8);
    if (na == 0) return;   // warp-uniform: this warp owns no row of the tile
#pragma unroll 2
    for (int q = 0; q < qb; ++q) {
        const int alo = TRI == TRI_LOWER ? q / 16 : 0;       // rows >= q only
        const int ahi = TRI == TRI_UPPER ? q / 16 : A - 1;   // rows <= q only
        float2 l[A], y[B];
#pragma unroll
        for (int a = 0; a < A; ++a) l[a] = a < na && a >= alo && a <= ahi ? L[q][tr + 16 * a] : czero<float2>();
#pragma unroll
        for (int b = 0; b < B; ++b) y[b] = b < nb ? Y[q][tc + 8 * b] : czero<float2>();
#pragma unroll
        for (int a = 0; a < A; ++a) {
            if (a >= na) break;
            if (a < alo || a > ahi) continue;
#pragma unroll
            for (int b = 0; b < B; ++b)
                if (b < nb) cfma(acc.v[a][b], l[a], y[b]);
        }
    }
}

// d = a b + d on one 8 x 8 x 4 FP64 block (warp-wide; a: this lane's entry
// of the 8 x 4 row-major left block, b: of the 4 x 8 column-major right
// block, d: this lane's two entries of the 8 x 8 result)
__device__ __forceinline__ void dmma_884(double a, double b, double &d0, double &d1) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// complex128: per 4 pivots and per 8 x 8 block, four FP64 matrix
// instructions (Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br); a lane loads one
// complex entry of each left and right fragment.  Pivots q >= qb enter as
// zeros.
template <int TRI, int RT, int B>
__device__ __forceinline__ void tile_mma_p(const double2 (*L)[RT + SPAD], const double2 (*Y)[8 * B + SPAD], int qb,
                                           TileAcc<double2, RT, B> &acc, int rows, int rn, int lt) {
    constexpr int NRB = RT / 32;
    const int w = lt >> 5, lane = lt & 31;
    const int nb = min(B, (rn + 7) / 8);
    for (int k0 = 0; k0 < qb; k0 += 4) {
        const int kk = k0 + (lane & 3);
        const bool kin = kk < qb;
        double2 bf[B];
#pragma unroll
        for (int b = 0; b < B; ++b) bf[b] = kin && b < nb ? Y[kk][8 * b + (lane >> 2)] : czero<double2>();
#pragma unroll
        for (int i = 0; i < NRB; ++i) {
            const int rb = w + 4 * i;   // row block: rows 8 rb .. 8 rb + 7
            if (8 * rb >= rows) break;   // warp-uniform
            if (TRI == TRI_UPPER && 8 * rb > k0 + 3) continue;   // rows <= q only
            if (TRI == TRI_LOWER && 8 * rb + 7 < k0) continue;   // rows >= q only
            const double2 af = kin ? L[kk][8 * rb + (lane >> 2)] : czero<double2>();
#pragma unroll
            for (int b = 0; b < B; ++b) {
                if (b >= nb) break;
                double2 &d0 = acc.v[i][2 * b], &d1 = acc.v[i][2 * b + 1];
                dmma_884(af.x, bf[b].x, d0.x, d1.x);
                dmma_884(-af.y, bf[b].y, d0.x, d1.x);
                dmma_884(af.x, bf[b].y, d0.y, d1.y);
                dmma_884(af.y, bf[b].x, d0.y, d1.y);
            }
        }
    }
}

template <int TRI = 0, class C, int RT, int B>
__device__ __forceinline__ void tile_mma(const SolveSmem<C, RT, B> &sm, int qb, TileAcc<C, RT, B> &acc, int rows,
                                         int rn) {
    tile_mma_p<TRI, RT, B>(sm.L, sm.Y, qb, acc, rows, rn, threadIdx.x);
}

// row_ptr(row)[col] -= acc for the thread's rows (< rows) and columns (< rn)
template <class C, int RT, int B, class RowPtr>
__device__ __forceinline__ void sub_acc(RowPtr row_ptr, int rows, int rn, const TileAcc<C, RT, B> &acc) {
    for_acc(acc, rows, rn, threadIdx.x, [&](int row, int col, const C &v) {
        C *x = row_ptr(row);
        x[col] = csub(x[col], v);
    });
}

// Y[q][r] = row_ptr(q)[r] for q < qb, r < rn (entries outside: as above)
template <class C, int TC, class RowPtr>
__device__ __forceinline__ void stage_rows_p(C (*Y)[TC + SPAD], RowPtr row_ptr, int qb, int rn, int lt, int nt) {
    for (int t = lt; t < qb * TC; t += nt) {
        const int q = t / TC, r = t % TC;
        if (r < rn) cp_async_elem(&Y[q][r], row_ptr(q) + r);
    }
}
template <class C, int RT, int B, class RowPtr>
__device__ __forceinline__ void stage_rows(SolveSmem<C, RT, B> &sm, RowPtr row_ptr, int qb, int rn) {
    stage_rows_p<C, 8 * B>(sm.Y, row_ptr, qb, rn, threadIdx.x, NT);
}

// false when right-hand sides r0 .. r0 + rn - 1 are zero throughout node v's
// subtree (forward-pass pruning mask; no mask: always true)
template <class R>
__device__ __forceinline__ bool live(const SolveArgs<R> &a, int v, int r0, int rn) {
    if (!a.mask) return true;
    const unsigned char *m = a.mask + (size_t)v * a.mask_nch;
    for (int g = r0 >> 5; g <= (r0 + rn - 1) >> 5; ++g)
        if (m[g]) return true;
    return false;
}

// false when right-hand side `col` is zero throughout node v's subtree
template <class R>
__device__ __forceinline__ bool col_live(const SolveArgs<R> &a, int v, int col) {
    return !a.mask || a.mask[(size_t)v * a.mask_nch + (col >> 5)];
}

// matrix handled by this CTA: blockIdx.z indexes the launch's matrix list
template <class R>
__device__ __forceinline__ size_t solve_matrix(const SolveArgs<R> &a) {
    return a.fmap ? (size_t)a.fmap[blockIdx.z] : (size_t)blockIdx.z;
}
// slot of x and of the workspace w used by this CTA
template <class R>
__device__ __forceinline__ size_t solve_slot(const SolveArgs<R> &a) {
    return a.xmap ? (size_t)a.xmap[blockIdx.z] : solve_matrix(a);
}

template <class R>
struct Ctx {
    using C = cplx<R>;
    int node, f, s, rn;
    const C *F;
    const int *vars;
    C *X;   // this slice of x; pivot rows are solved in place here
    C *W;   // this node's update vector: ring row i (front position s + i)
};

template <class R, int TC>
__device__ __forceinline__ Ctx<R> make_ctx(const SolveArgs<R> &a, int lvl_first, int chunk, int pos = -1) {
    using C = cplx<R>;
    Ctx<R> c;
    c.node = a.s.lvl_nodes[lvl_first + (pos < 0 ? (int)blockIdx.y : pos)];
    c.f = a.s.nfront[c.node];
    c.s = a.s.npiv[c.node];
    const int r0 = chunk * TC;
    c.rn = min(TC, a.nrhs - r0);
    const size_t fz = solve_matrix(a), xz = solve_slot(a);
    c.F = reinterpret_cast<const C *>(a.front) + fz * a.s.front_total + a.s.front_off[c.node];
    c.vars = a.s.vars + a.s.var_off[c.node];
    c.X = reinterpret_cast<C *>(a.x) + xz * (size_t)a.s.n * a.ldr + r0;
    c.W = reinterpret_cast<C *>(a.w) + xz * (size_t)a.s.rhs_total * a.ldr + r0 + (size_t)a.s.rhs_off[c.node] * a.ldr;
    return c;
}

// The pivot rows of this front's slice of x receive the children's update
// vectors (W0, W1: NULL for a child that is absent or pruned); with implicit
// spike right-hand sides they become b + the updates, x not being read
// (it is not cleared before the solve).
template <class R>
__device__ __forceinline__ void pivot_rhs(const SolveArgs<R> &a, const Ctx<R> &c, const int *inv, const cplx<R> *W0,
                                          const cplx<R> *W1, int r0, size_t ldr) {
    using C = cplx<R>;
    const bool implicit = a.spike_k != nullptr;
    if (!(W0 || W1 || implicit)) return;   // CTA-uniform
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const C amp = implicit ? cconv<C>(a.spike_amp[solve_matrix(a)]) : czero<C>();
    for (int i = warp; i < c.s; i += NT / 32) {
        const int q0 = W0 ? inv[i] : -1, q1 = W1 ? inv[c.f + i] : -1;
        if (!implicit && q0 < 0 && q1 < 0) continue;
        const int row = c.vars[i];
        for (int r = lane; r < c.rn; r += 32) {
            C v = czero<C>();
            if (q0 >= 0) v = cadd(v, W0[(size_t)q0 * ldr + r]);
            if (q1 >= 0) v = cadd(v, W1[(size_t)q1 * ldr + r]);
            C &x = c.X[(size_t)row * ldr + r];
            x = implicit ? (a.spike_k[r0 + r] == row ? cadd(amp, v) : v) : cadd(x, v);
        }
    }
    __syncthreads();
}

// Forward pass, pivot part: add the children's update vectors (gathered by
// the extend-add inverse maps) into x at this front's pivots, then solve the
// pivot rows in place in x, 32-pivot block by block.
template <class R, bool TRANS, int RT, int B>
__global__ void __launch_bounds__(NT) k_fwd_piv(SolveArgs<R> a, int lvl_first, int fused) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SolveSmem<C, RT, B> &sm = *reinterpret_cast<SolveSmem<C, RT, B> *>(smem_raw);
    constexpr int TC = 8 * B;
    const Ctx<R> c = make_ctx<R, TC>(a, lvl_first, blockIdx.x);
    if (c.rn <= 0) return;
    const int r0 = blockIdx.x * TC;
    if (!live(a, c.node, r0, c.rn)) return;   // y and the update vector are zero
    (void)fused;
    const int *inv = a.s.inv + a.s.inv_off[c.node];
    const size_t xz = solve_slot(a);
    const C *Wall = reinterpret_cast<const C *>(a.w) + xz * (size_t)a.s.rhs_total * a.ldr + r0;
    const int c0 = a.s.child0[c.node], c1 = a.s.child1[c.node];
    const C *W0 = c0 >= 0 && live(a, c0, r0, c.rn) ? Wall + (size_t)a.s.rhs_off[c0] * a.ldr : nullptr;
    const C *W1 = c1 >= 0 && live(a, c1, r0, c.rn) ? Wall + (size_t)a.s.rhs_off[c1] * a.ldr : nullptr;
    const size_t ldr = a.ldr;

    pivot_rhs(a, c, inv, W0, W1, r0, ldr);   // (the ring part is k_fwd_ring's)

    auto xrow = [&](int k) { return c.X + (size_t)c.vars[k] * ldr; };
    // M x = b with row exchanges: block k0's right-hand-side rows are taken
    // in pivot order (prow[q]: the block row at pivot position q), y is
    // written in pivot order (rows of L' below the block stay in equation
    // order until their own block)
    __shared__ unsigned char prow[SNB];
    const bool pv = !TRANS && a.pivsrc;
    const unsigned char *psrc = pv ? a.pivsrc + solve_matrix(a) * (size_t)a.s.n : nullptr;
    TileAcc<C, RT, B> acc;
    for (int k0 = 0; k0 < c.s; k0 += SNB) {
        const int kb = min(SNB, c.s - k0);
        if (pv) {   // the previous block's reads of prow ended before its staged_sync
            if (threadIdx.x < kb) prow[threadIdx.x] = psrc[c.vars[k0 + threadIdx.x]];
            __syncthreads();
        }
        stage_dinv<C, true, TRANS, RT, B>(sm, c.F, c.f, k0, kb);
        stage_rows(sm, [&](int q) { return xrow(k0 + (pv ? prow[q] : q)); }, kb, c.rn);
        staged_sync();
        zero_acc(acc);
        tile_mma<TRI_LOWER>(sm, kb, acc, kb, c.rn);   // y_b = Dinv w_b
        __syncthreads();
        for_acc(acc, kb, c.rn, threadIdx.x, [&](int row, int col, const C &v) { sm.Y[row][col] = v; });
        __syncthreads();
        for (int t = threadIdx.x; t < kb * TC; t += NT) {
            const int q = t / TC, r = t % TC;
            if (r < c.rn) xrow(k0 + q)[r] = sm.Y[q][r];
        }
        for (int i0 = k0 + kb; i0 < c.s; i0 += RT) {
            const int rows = min(RT, c.s - i0);
            stage_factor<C, TRANS, RT, B>(sm, c.F, c.f, i0, rows, k0, kb);
            staged_sync();
            zero_acc(acc);
            tile_mma(sm, kb, acc, rows, c.rn);
            sub_acc([&](int row) { return xrow(i0 + row); }, rows, c.rn, acc);
            __syncthreads();
        }
    }
}

// Forward pass, ring part: update vector = children's update vectors at the
// ring rows - L'(ring, pivots) y, 64-row tiles of the ring over many CTAs;
// blockIdx.x = chunk + nchunk * tile
template <class R, bool TRANS, int RT, int B>
__global__ void __launch_bounds__(NT) k_fwd_ring(SolveArgs<R> a, int lvl_first, int nchunk) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SolveSmem<C, RT, B> &sm = *reinterpret_cast<SolveSmem<C, RT, B> *>(smem_raw);
    constexpr int TC = 8 * B;
    const int chunk = blockIdx.x % nchunk, tile = blockIdx.x / nchunk;
    const Ctx<R> c = make_ctx<R, TC>(a, lvl_first, chunk);
    const int i0 = c.s + tile * RT;
    if (c.rn <= 0 || i0 >= c.f) return;
    if (!live(a, c.node, chunk * TC, c.rn)) return;   // the update vector is zero (never read)
    const int rows = min(RT, c.f - i0);
    const size_t ldr = a.ldr;
    TileAcc<C, RT, B> acc;
    zero_acc(acc);
    for (int q0 = 0; q0 < c.s; q0 += SNB) {
        const int qb = min(SNB, c.s - q0);
        stage_factor<C, TRANS, RT, B>(sm, c.F, c.f, i0, rows, q0, qb);
        stage_rows(sm, [&](int q) { return c.X + (size_t)c.vars[q0 + q] * ldr; }, qb, c.rn);
        staged_sync();
        tile_mma(sm, qb, acc, rows, c.rn);
        __syncthreads();
    }
    // w = (children's update vectors at the ring rows) - L'(ring, piv) y
    const int *inv = a.s.inv + a.s.inv_off[c.node];
    const C *Wall = reinterpret_cast<const C *>(a.w) + solve_slot(a) * a.s.rhs_total * a.ldr + chunk * TC;
    const int c0 = a.s.child0[c.node], c1 = a.s.child1[c.node];
    const C *W0 = c0 >= 0 && live(a, c0, chunk * TC, c.rn) ? Wall + (size_t)a.s.rhs_off[c0] * a.ldr : nullptr;
    const C *W1 = c1 >= 0 && live(a, c1, chunk * TC, c.rn) ? Wall + (size_t)a.s.rhs_off[c1] * a.ldr : nullptr;
    for_acc(acc, rows, c.rn, threadIdx.x, [&](int row, int r, const C &v) {
        const int i = i0 + row;
        const int q0 = W0 ? inv[i] : -1, q1 = W1 ? inv[c.f + i] : -1;
        C g = czero<C>();
        if (q0 >= 0) g = cadd(g, W0[(size_t)q0 * ldr + r]);
        if (q1 >= 0) g = cadd(g, W1[(size_t)q1 * ldr + r]);
        c.W[(size_t)(i - c.s) * ldr + r] = csub(g, v);
    });
}

// Backward pass, ring part: x[pivots] -= U'(pivots, ring) x[ring]
// (final values of the ancestors' variables); blockIdx.x = chunk + nchunk * tile
template <class R, bool TRANS, int RT, int B>
__global__ void __launch_bounds__(NT) k_bwd_ring(SolveArgs<R> a, int lvl_first, int nchunk) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SolveSmem<C, RT, B> &sm = *reinterpret_cast<SolveSmem<C, RT, B> *>(smem_raw);
    constexpr int TC = 8 * B;
    const int chunk = blockIdx.x % nchunk, tile = blockIdx.x / nchunk;
    const Ctx<R> c = make_ctx<R, TC>(a, lvl_first, chunk);
    const int i0 = tile * RT;
    if (c.rn <= 0 || i0 >= c.s || c.f == c.s) return;
    const int rows = min(RT, c.s - i0);
    const size_t ldr = a.ldr;
    TileAcc<C, RT, B> acc;
    zero_acc(acc);
    for (int j0 = c.s; j0 < c.f; j0 += SNB) {
        const int jb = min(SNB, c.f - j0);
        stage_factor<C, TRANS, RT, B>(sm, c.F, c.f, i0, rows, j0, jb);
        stage_rows(sm, [&](int q) { return c.X + (size_t)c.vars[j0 + q] * ldr; }, jb, c.rn);
        staged_sync();
        tile_mma(sm, jb, acc, rows, c.rn);
        __syncthreads();
    }
    // y = 0 at the pivot rows in the right-hand sides the pruned forward
    // pass skipped for this front (x is not cleared there when the
    // right-hand sides are implicit spikes)
    for_acc(acc, rows, c.rn, threadIdx.x, [&](int row, int col, const C &v) {
        C &x = c.X[(size_t)c.vars[i0 + row] * ldr + col];
        x = csub(a.spike_k && !col_live(a, c.node, chunk * TC + col) ? czero<C>() : x, v);
    });
}

// Backward pass, pivot part: block by block from the last, x_b = Dinv t_b in
// place in x, then t_above -= U'(above, b) x_b.
template <class R, bool TRANS, int RT, int B>
__global__ void __launch_bounds__(NT) k_bwd_piv(SolveArgs<R> a, int lvl_first, int fused) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SolveSmem<C, RT, B> &sm = *reinterpret_cast<SolveSmem<C, RT, B> *>(smem_raw);
    constexpr int TC = 8 * B;
    const Ctx<R> c = make_ctx<R, TC>(a, lvl_first, blockIdx.x);
    if (c.rn <= 0) return;
    (void)fused;
    const size_t ldr = a.ldr;
    auto xrow = [&](int k) { return c.X + (size_t)c.vars[k] * ldr; };
    if (c.f == c.s && a.spike_k) {
        // no ring (k_bwd_ring did not set y): y = 0 at the pivot rows in the
        // right-hand sides the pruned forward pass skipped for this front
        for (int t = threadIdx.x; t < c.s * TC; t += NT) {
            const int q = t / TC, r = t % TC;
            if (r < c.rn && !col_live(a, c.node, blockIdx.x * TC + r)) xrow(q)[r] = czero<C>();
        }
        __syncthreads();
    }
    // M^T x = b with row exchanges: the block's result comes out in pivot
    // order and is scattered to equation order (prow[q]: the block row at
    // pivot position q), where the updates of the blocks above read it
    __shared__ unsigned char prow[SNB];
    const bool pv = TRANS && a.pivsrc;
    const unsigned char *psrc = pv ? a.pivsrc + solve_matrix(a) * (size_t)a.s.n : nullptr;
    TileAcc<C, RT, B> acc;
    const int nblk = (c.s + SNB - 1) / SNB;
    for (int b = nblk - 1; b >= 0; --b) {
        const int k0 = b * SNB, kb = min(SNB, c.s - k0);
        if (pv && threadIdx.x < kb) prow[threadIdx.x] = psrc[c.vars[k0 + threadIdx.x]];   // read after staged_sync
        stage_dinv<C, false, TRANS, RT, B>(sm, c.F, c.f, k0, kb);
        stage_rows(sm, [&](int q) { return xrow(k0 + q); }, kb, c.rn);
        staged_sync();
        zero_acc(acc);
        tile_mma<TRI_UPPER>(sm, kb, acc, kb, c.rn);   // x_b = Dinv t_b
        __syncthreads();
        for_acc(acc, kb, c.rn, threadIdx.x, [&](int row, int col, const C &v) { sm.Y[pv ? prow[row] : row][col] = v; });
        __syncthreads();
        for (int t = threadIdx.x; t < kb * TC; t += NT) {
            const int q = t / TC, r = t % TC;
            if (r < c.rn) xrow(k0 + q)[r] = sm.Y[q][r];
        }
        for (int i0 = 0; i0 < k0; i0 += RT) {
            const int rows = min(RT, k0 - i0);
            stage_factor<C, TRANS, RT, B>(sm, c.F, c.f, i0, rows, k0, kb);
            staged_sync();
            zero_acc(acc);
            tile_mma(sm, kb, acc, rows, c.rn);
            sub_acc([&](int row) { return xrow(i0 + row); }, rows, c.rn, acc);
            __syncthreads();
        }
    }
}

// (The complex128 small-front kernels are held to 80 registers, six CTAs per
// SM: measured on the leaf levels they stall on global loads first, so more
// resident warps pay; the complex64 ones need fewer registers anyway.)
//
// Forward pass of a whole front whose pivots fit one 32-pivot block (the
// small fronts of the lower levels): the children's update vectors are added
// into x at the pivots, y = Dinv x_piv is formed in shared memory and written
// back to x, and the update vector w = (children's update vectors at the
// ring rows) - L'(ring, pivots) y follows tile by tile with y kept in shared
// memory -- k_fwd_piv and k_fwd_ring in one CTA, y read once.
// wofs >= 0: the CTA's (front position, slice) is work[wofs + blockIdx.x],
// the live pairs of a pruned pass; wofs < 0: (blockIdx.y, blockIdx.x).
template <class R, bool TRANS, int B>
__global__ void __launch_bounds__(NT, sizeof(R) == 8 ? 6 : 1) k_fwd_small(SolveArgs<R> a, int lvl_first, int wofs) {
    using C = cplx<R>;
    constexpr int RT = 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SolveSmem<C, RT, B> &sm = *reinterpret_cast<SolveSmem<C, RT, B> *>(smem_raw);
    constexpr int TC = 8 * B;
    const int2 wk = wofs >= 0 ? a.work[wofs + blockIdx.x] : make_int2((int)blockIdx.y, (int)blockIdx.x);
    const Ctx<R> c = make_ctx<R, TC>(a, lvl_first, wk.y, wk.x);
    if (c.rn <= 0) return;
    const int r0 = wk.y * TC;
    if (!live(a, c.node, r0, c.rn)) return;   // y and the update vector are zero
    const int *inv = a.s.inv + a.s.inv_off[c.node];
    const size_t xz = solve_slot(a);
    const C *Wall = reinterpret_cast<const C *>(a.w) + xz * (size_t)a.s.rhs_total * a.ldr + r0;
    const int c0 = a.s.child0[c.node], c1 = a.s.child1[c.node];
    const C *W0 = c0 >= 0 && live(a, c0, r0, c.rn) ? Wall + (size_t)a.s.rhs_off[c0] * a.ldr : nullptr;
    const C *W1 = c1 >= 0 && live(a, c1, r0, c.rn) ? Wall + (size_t)a.s.rhs_off[c1] * a.ldr : nullptr;
    const size_t ldr = a.ldr;
    const int s = c.s;   // <= SNB (launch condition)

    pivot_rhs(a, c, inv, W0, W1, r0, ldr);
    // M x = b with row exchanges: the pivot rows' right-hand sides are taken
    // in pivot order (prow[q]: the front row at pivot position q)
    __shared__ unsigned char prow[SNB];
    const bool pv = !TRANS && a.pivsrc;
    if (pv) {
        if (threadIdx.x < s) prow[threadIdx.x] = a.pivsrc[solve_matrix(a) * (size_t)a.s.n + c.vars[threadIdx.x]];
        __syncthreads();
    }
    TileAcc<C, RT, B> acc;
    if (s > 0) {
        stage_dinv<C, true, TRANS, RT, B>(sm, c.F, c.f, 0, s);
        stage_rows(sm, [&](int q) { return c.X + (size_t)c.vars[pv ? prow[q] : q] * ldr; }, s, c.rn);
        staged_sync();
        zero_acc(acc);
        tile_mma<TRI_LOWER>(sm, s, acc, s, c.rn);   // y = Dinv x_piv
        __syncthreads();
        for_acc(acc, s, c.rn, threadIdx.x, [&](int row, int col, const C &v) { sm.Y[row][col] = v; });
        __syncthreads();
        for (int t = threadIdx.x; t < s * TC; t += NT) {
            const int q = t / TC, r = t % TC;
            if (r < c.rn) c.X[(size_t)c.vars[q] * ldr + r] = sm.Y[q][r];
        }
    }
    // w over the ring rows, 32-row tiles, y staying in sm.Y
    for (int i0 = s; i0 < c.f; i0 += RT) {
        const int rows = min(RT, c.f - i0);
        stage_factor<C, TRANS, RT, B>(sm, c.F, c.f, i0, rows, 0, s);
        staged_sync();
        zero_acc(acc);
        tile_mma(sm, s, acc, rows, c.rn);
        for_acc(acc, rows, c.rn, threadIdx.x, [&](int row, int r, const C &v) {
            const int i = i0 + row;
            const int q0 = W0 ? inv[i] : -1, q1 = W1 ? inv[c.f + i] : -1;
            C g = czero<C>();
            if (q0 >= 0) g = cadd(g, W0[(size_t)q0 * ldr + r]);
            if (q1 >= 0) g = cadd(g, W1[(size_t)q1 * ldr + r]);
            c.W[(size_t)(i - s) * ldr + r] = csub(g, v);
        });
        __syncthreads();   // sm.L is staged again for the next tile
    }
}

// Backward pass of a whole front whose pivots fit one 32-pivot block (the
// small fronts of the lower levels): t = y - U'(pivots, ring) x[ring] with
// the product accumulated in registers over 32-column ring blocks, t placed
// in shared memory, then x_piv = Dinv t -- k_bwd_ring and k_bwd_piv in one
// CTA, without writing t to x in between.
template <class R, bool TRANS, int B>
__global__ void __launch_bounds__(NT, sizeof(R) == 8 ? 6 : 1) k_bwd_small(SolveArgs<R> a, int lvl_first) {
    using C = cplx<R>;
    constexpr int RT = 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SolveSmem<C, RT, B> &sm = *reinterpret_cast<SolveSmem<C, RT, B> *>(smem_raw);
    constexpr int TC = 8 * B;
    const Ctx<R> c = make_ctx<R, TC>(a, lvl_first, blockIdx.x);
    if (c.rn <= 0 || c.s == 0) return;
    const size_t ldr = a.ldr;
    const int s = c.s;   // <= SNB (launch condition)
    // M^T x = b with row exchanges: the result comes out in pivot order and
    // is scattered to equation order (prow[q]: the front row at pivot
    // position q; read after the staged_sync below)
    __shared__ unsigned char prow[SNB];
    const bool pv = TRANS && a.pivsrc;
    if (pv && threadIdx.x < s) prow[threadIdx.x] = a.pivsrc[solve_matrix(a) * (size_t)a.s.n + c.vars[threadIdx.x]];
    TileAcc<C, RT, B> acc;
    zero_acc(acc);
    for (int j0 = s; j0 < c.f; j0 += SNB) {
        const int jb = min(SNB, c.f - j0);
        stage_factor<C, TRANS, RT, B>(sm, c.F, c.f, 0, s, j0, jb);
        stage_rows(sm, [&](int q) { return c.X + (size_t)c.vars[j0 + q] * ldr; }, jb, c.rn);
        staged_sync();
        tile_mma(sm, jb, acc, s, c.rn);
        __syncthreads();
    }
    // t = y - acc in sm.Y (row q of the next product's right operand = pivot
    // q); y = 0 where the pruned forward pass skipped the front (its rows of
    // x are not cleared when the right-hand sides are implicit spikes)
    if (a.spike_k) {   // y = 0 in the right-hand sides the pruned forward pass skipped
        for (int t = threadIdx.x; t < s * TC; t += NT) {
            const int q = t / TC, r = t % TC;
            if (r >= c.rn) continue;
            if (col_live(a, c.node, blockIdx.x * TC + r)) cp_async_elem(&sm.Y[q][r], c.X + (size_t)c.vars[q] * ldr + r);
            else sm.Y[q][r] = czero<C>();
        }
    } else {
        stage_rows(sm, [&](int q) { return c.X + (size_t)c.vars[q] * ldr; }, s, c.rn);
    }
    stage_dinv<C, false, TRANS, RT, B>(sm, c.F, c.f, 0, s);
    staged_sync();
    for_acc(acc, s, c.rn, threadIdx.x, [&](int row, int col, const C &v) { sm.Y[row][col] = csub(sm.Y[row][col], v); });
    __syncthreads();
    zero_acc(acc);
    tile_mma<TRI_UPPER>(sm, s, acc, s, c.rn);   // x_piv = Dinv t
    for_acc(acc, s, c.rn, threadIdx.x,
            [&](int row, int col, const C &v) { c.X[(size_t)c.vars[pv ? prow[row] : row] * ldr + col] = v; });
}

template <class R, int RT, int B>
static size_t solve_smem() { return sizeof(SolveSmem<cplx<R>, RT, B>); }

template <class R, int RT, int B>
static void set_attrs() {
    static bool done = false;
    if (done) return;
    const int sm = (int)solve_smem<R, RT, B>();
    cudaFuncSetAttribute((const void *)k_fwd_piv<R, false, RT, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute((const void *)k_fwd_piv<R, true, RT, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute((const void *)k_fwd_ring<R, false, RT, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute((const void *)k_fwd_ring<R, true, RT, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute((const void *)k_bwd_ring<R, false, RT, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute((const void *)k_bwd_ring<R, true, RT, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute((const void *)k_bwd_piv<R, false, RT, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute((const void *)k_bwd_piv<R, true, RT, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (RT == 32) {
        cudaFuncSetAttribute((const void *)k_bwd_small<R, false, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute((const void *)k_bwd_small<R, true, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute((const void *)k_fwd_small<R, false, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute((const void *)k_fwd_small<R, true, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    }
    done = true;
}

static int env_int(const char *name) {
    const char *v = std::getenv(name);
    return v ? std::atoi(v) : 0;
}

// Tile height of a level: 32-row tiles wherever the level has many fronts
// (measured on 841 x 227: 14 % less substitution time than 64-row tiles,
// the gain coming from the 4096 .. 16-front levels), 64-row tiles on the
// top levels of at most four fronts, where the tiles of one front are the
// parallelism.  GM_SOLVE_RT=32 / 64 forces one height on every level.
static int level_rt(const LevelInfo &L) {
    static const int forced = env_int("GM_SOLVE_RT");
    if (forced == 32 || forced == 64) return forced;
    return L.count > 4 ? 32 : 64;
}

// Right-hand-side slice width (8 B).  Measured on 841 x 227 with 100
// right-hand sides: 32 / 40 / 56 columns give 36.6 / 36.6 / 38.0 ms per
// complex128 substitution and 19.9 / 19.1 / 19.8 ms per complex64 one, so
// the lower levels are not bound by re-reading the factors per slice.
// GM_SOLVE_B=4 / 5 forces 32 / 40.
template <class R>
static int slice_b(int nrhs) {
    static const int forced = env_int("GM_SOLVE_B");
    if (forced == 4 || forced == 5) return forced;
    return (sizeof(R) == 4 && nrhs > 32) ? 5 : 4;
}

template <class R>
static int solve_nfz(const SolveArgs<R> &a) { return a.fmap ? a.nfz : a.nf; }

template <class R, int RT, int B>
static void forward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    set_attrs<R, RT, B>();
    const size_t smem = solve_smem<R, RT, B>();
    const int nchunk = (a.nrhs + 8 * B - 1) / (8 * B);
    static const bool no_small = env_int("GM_NO_FWD_SMALL") != 0;
    if (RT == 32 && L.max_piv <= SNB && !no_small) {   // one pivot block per front: fused pivot + ring kernel
        if (a.work && a.work_w[L.index] == 8 * B) {   // pruned pass: only the live (front, slice) pairs
            const int wofs = a.work_off[L.index];
            const int nlive = a.work_off[L.index + 1] - wofs;
            if (nlive == 0) return;
            dim3 g(nlive, 1, solve_nfz(a));
            if (a.trans) (k_fwd_small<R, true, B><<<g, NT, smem, st>>>(a, L.first, wofs), note_launch());
            else (k_fwd_small<R, false, B><<<g, NT, smem, st>>>(a, L.first, wofs), note_launch());
            return;
        }
        for_level_pieces(L, [&](int first, int count) {
            dim3 g(nchunk, count, solve_nfz(a));
            if (a.trans) (k_fwd_small<R, true, B><<<g, NT, smem, st>>>(a, first, -1), note_launch());
            else (k_fwd_small<R, false, B><<<g, NT, smem, st>>>(a, first, -1), note_launch());
        });
        return;
    }
    const int fused = 0;   // separate ring kernel: more parallelism per level
    for_level_pieces(L, [&](int first, int count) {
        dim3 g1(nchunk, count, solve_nfz(a));
        if (a.trans) (k_fwd_piv<R, true, RT, B><<<g1, NT, smem, st>>>(a, first, fused), note_launch());
        else (k_fwd_piv<R, false, RT, B><<<g1, NT, smem, st>>>(a, first, fused), note_launch());
    });
    if (L.max_ring > 0) {
        for_level_pieces(L, [&](int first, int count) {
            dim3 g2(nchunk * ((L.max_ring + RT - 1) / RT), count, solve_nfz(a));
            if (a.trans) (k_fwd_ring<R, true, RT, B><<<g2, NT, smem, st>>>(a, first, nchunk), note_launch());
            else (k_fwd_ring<R, false, RT, B><<<g2, NT, smem, st>>>(a, first, nchunk), note_launch());
        });
    }
}

template <class R, int RT, int B>
static void backward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    set_attrs<R, RT, B>();
    const size_t smem = solve_smem<R, RT, B>();
    const int nchunk = (a.nrhs + 8 * B - 1) / (8 * B);
    static const bool no_small = env_int("GM_NO_BWD_SMALL") != 0;
    if (RT == 32 && L.max_piv <= SNB && !no_small) {   // one pivot block per front: fused ring + pivot kernel
        for_level_pieces(L, [&](int first, int count) {
            dim3 g(nchunk, count, solve_nfz(a));
            if (a.trans) (k_bwd_small<R, true, B><<<g, NT, smem, st>>>(a, first), note_launch());
            else (k_bwd_small<R, false, B><<<g, NT, smem, st>>>(a, first), note_launch());
        });
        return;
    }
    const int fused = 0;
    if (L.max_ring > 0) {
        for_level_pieces(L, [&](int first, int count) {
            dim3 g1(nchunk * ((L.max_piv + RT - 1) / RT), count, solve_nfz(a));
            if (a.trans) (k_bwd_ring<R, true, RT, B><<<g1, NT, smem, st>>>(a, first, nchunk), note_launch());
            else (k_bwd_ring<R, false, RT, B><<<g1, NT, smem, st>>>(a, first, nchunk), note_launch());
        });
    }
    for_level_pieces(L, [&](int first, int count) {
        dim3 g2(nchunk, count, solve_nfz(a));
        if (a.trans) (k_bwd_piv<R, true, RT, B><<<g2, NT, smem, st>>>(a, first, fused), note_launch());
        else (k_bwd_piv<R, false, RT, B><<<g2, NT, smem, st>>>(a, first, fused), note_launch());
    });
}

template <class R, int B>
static void level_pass(bool fwd, const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    if (level_rt(L) == 32) {
        if (fwd) forward_level<R, 32, B>(a, L, st);
        else backward_level<R, 32, B>(a, L, st);
    } else {
        if (fwd) forward_level<R, 64, B>(a, L, st);
        else backward_level<R, 64, B>(a, L, st);
    }
}

template <class R, int B>
static void level_pass_rt(bool fwd, int rt, const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    if (rt == 32) {
        if (fwd) forward_level<R, 32, B>(a, L, st);
        else backward_level<R, 32, B>(a, L, st);
    } else {
        if (fwd) forward_level<R, 64, B>(a, L, st);
        else backward_level<R, 64, B>(a, L, st);
    }
}

// The level's tile height and slice width: the autotuned choice when the
// engine holds one (a.lvl_cfg, per level: forward rt, forward B, backward
// rt, backward B; 0 = the default rule), else the default rules above.
template <class R>
static void dispatch(bool fwd, const SolveArgs<R> &a_in, const LevelInfo &L, cudaStream_t st) {
    if (L.count == 0 || solve_nfz(a_in) <= 0) return;
    SolveArgs<R> a = a_in;
    if (!level_pivots<R>(L)) a.pivsrc = nullptr;   // no row exchanges on this level
    if (a.lvl_cfg) {
        const int *c = a.lvl_cfg + 4 * L.index + (fwd ? 0 : 2);
        const int rt = c[0] ? c[0] : level_rt(L), b = c[1] ? c[1] : slice_b<R>(a.nrhs);
        if (b == 5) level_pass_rt<R, 5>(fwd, rt, a, L, st);
        else level_pass_rt<R, 4>(fwd, rt, a, L, st);
        return;
    }
    if (slice_b<R>(a.nrhs) == 5) level_pass<R, 5>(fwd, a, L, st);
    else level_pass<R, 4>(fwd, a, L, st);
}

template <class R>
void launch_solve_forward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    dispatch<R>(true, a, L, st);
}

template <class R>
void launch_solve_backward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    dispatch<R>(false, a, L, st);
}

// Sets the shared-memory attribute of every substitution kernel variant,
// which also loads each kernel (CUDA loads modules and functions lazily, on
// first use, and a load takes device memory): a caller that must not
// allocate once solving has begun calls this beforehand.
void preload_solve_kernels() {
    set_attrs<double, 32, 4>();
    set_attrs<double, 64, 4>();
    set_attrs<double, 32, 5>();
    set_attrs<double, 64, 5>();
    set_attrs<float, 32, 4>();
    set_attrs<float, 64, 4>();
    set_attrs<float, 32, 5>();
    set_attrs<float, 64, 5>();
}

int solve_slice_width(int nrhs, bool fp64) { return 8 * (fp64 ? slice_b<double>(nrhs) : slice_b<float>(nrhs)); }
int solve_level_rt(const LevelInfo &L) { return level_rt(L); }

template void launch_solve_forward_level<double>(const SolveArgs<double> &, const LevelInfo &, cudaStream_t);
template void launch_solve_forward_level<float>(const SolveArgs<float> &, const LevelInfo &, cudaStream_t);
template void launch_solve_backward_level<double>(const SolveArgs<double> &, const LevelInfo &, cudaStream_t);
template void launch_solve_backward_level<float>(const SolveArgs<float> &, const LevelInfo &, cudaStream_t);

}  // namespace gm
