// K2-K4: numeric multifrontal LU of one elimination-tree level, batched
// over every front of the level and every frequency (the replacement of
// umfpack_zi_numeric, src/AC/forward_shot_AC.c:61).
//
// Fronts live in HBM as dense column-major nfront x nfront complex blocks
// (one block per node per frequency).  A level is processed by
//   K2 gather   -- each front pulls its children's contribution blocks
//                  (extend-add by inverse maps: deterministic, no atomics),
//   K2 scatter  -- adds the operator entries owned by the front,
//   K3 diag     -- per NB-wide pivot block: LU of the diagonal block with
//                  threshold partial pivoting inside the block (static
//                  pivots as the last resort) and the inverses of its two
//                  triangles, factored once per front (the first block by
//                  k_diag, each later one by the first CTA of the preceding
//                  K4),
//   K3 panels   -- L21 = A21 U11^-1 and U12 = L11^-1 P A12 as products with
//                  those inverses (FP64 matrix instructions in complex128),
//   K4 update   -- rank-NB Schur update of the pivot rows and columns still
//                  to come, 64x64 tiles.
// K3/K4 alternate ceil(max_piv/NB) times per level.  After the last step a
// front holds L (unit lower) and U in its first npiv rows/columns -- except
// that each NB x NB diagonal block holds the INVERSES of its two triangles
// (what the substitution multiplies by) -- and its Schur complement (the
// contribution block) in the trailing block.  With row exchanges, the rows
// of a block's diagonal block and U part are in pivot order, its rows'
// multipliers of earlier blocks in equation order, and the block's
// permutation is in FactorArgs::pivsrc.
//
// Two fused kernels leave the same layout on the levels where they pay:
//   k_factor_small  fronts that fit shared memory whole (the lower levels):
//                   extend-add, entries, LU and Schur complement in one CTA;
//   k_factor_mid    fronts with at most NB pivots and at most 256 rows above
//                   those: after K2, one CTA factorises the pivot columns
//                   and applies the Schur update to the contribution block
//                   once, in place of K3 / K4 and the contribution GEMM.
// The remaining (upper) levels take the blocked K2-K4 sequence.
#include <cstdlib>
#include "kernels.cuh"
#include "cplx.cuh"
#include "async_copy.cuh"

namespace gm {

constexpr int NB = 32;       // pivot block width
constexpr int TILE = 64;     // Schur-update tile

constexpr int GATHER_COLS = 4;   // front columns per CTA of the extend-add gather
constexpr int TSTR = TILE + 2;   // padded row stride of staged 64-wide tiles (conflict-free 8 x 4 fragments)

// 64 x 64 complex output tile of a 256-thread CTA, in the layout of the
// product that fills it: complex64 with CUDA-core FMAs, thread t owning
// rows t % 16 + 16 i and columns t / 16 + 16 j (v[i][j]); complex128 on FP64
// matrix instructions (mma.sync m8n8k4 f64) on 8 x 8 blocks, warp w owning
// row blocks w % 4 and w % 4 + 4 of column blocks 4 (w / 4) .. 4 (w / 4) + 3
// (so a tile with few rows still keeps six of the eight warps busy), lane l
// row 8 rb + l / 4 and columns 8 cb + 2 (l % 4) + j of each owned block;
// v[4 rbi + cbi][j] for row block w % 4 + 4 rbi, column block 4 (w / 4) + cbi.
template <class C, bool MMA>
struct Tile64;
template <class C>
struct Tile64<C, false> {   // CUDA-core FMAs (complex64, or complex128 where short K suits them better)
    static constexpr int NI = 4, NJ = 4;
    C v[NI][NJ];
    __device__ __forceinline__ static int row(int i, int, int t) { return t % 16 + 16 * i; }
    __device__ __forceinline__ static int col(int, int j, int t) { return t / 16 + 16 * j; }
};
template <>
struct Tile64<double2, true> {   // FP64 matrix instructions
    static constexpr int NI = 8, NJ = 2;
    double2 v[NI][NJ];
    __device__ __forceinline__ static int row(int i, int, int t) {
        return 8 * ((t >> 5) % 4 + 4 * (i / 4)) + ((t & 31) >> 2);
    }
    __device__ __forceinline__ static int col(int i, int j, int t) {
        return 8 * (4 * ((t >> 5) / 4) + i % 4) + 2 * (t & 3) + j;
    }
};

// f(row, col, value) over the thread's entries of the tile
template <class C, bool MMA, class F>
__device__ __forceinline__ void for_tile64(Tile64<C, MMA> &acc, int t, F f) {
    using T = Tile64<C, MMA>;
#pragma unroll
    for (int i = 0; i < T::NI; ++i)
#pragma unroll
        for (int j = 0; j < T::NJ; ++j) f(T::row(i, j, t), T::col(i, j, t), acc.v[i][j]);
}

// acc += A B (NEG: acc -= A B) over k < kb, A(r, k) = As[k * ak + r * ar]
// for rows r < mrows, B(k, c) = Bs[k * bk + c * bc] for columns c < ncols
// (entries outside read as zero)
template <bool NEG, class C>
__device__ __forceinline__ void mma64(const C *As, int ak, int ar, const C *Bs, int bk, int bc, int kb, int mrows,
                                      int ncols, Tile64<C, false> &acc, int t) {
    const int tx = t % 16, ty = t / 16;
    for (int k = 0; k < kb; ++k) {
        C lv[4], uv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
            lv[i] = tx + 16 * i < mrows ? As[(size_t)k * ak + (size_t)(tx + 16 * i) * ar] : czero<C>();
#pragma unroll
        for (int j = 0; j < 4; ++j)
            uv[j] = ty + 16 * j < ncols ? Bs[(size_t)k * bk + (size_t)(ty + 16 * j) * bc] : czero<C>();
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (NEG) cfms(acc.v[i][j], lv[i], uv[j]);
                else cfma(acc.v[i][j], lv[i], uv[j]);
            }
    }
}

__device__ __forceinline__ void dmma_884(double a, double b, double &d0, double &d1) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <bool NEG>
__device__ __forceinline__ void mma64(const double2 *As, int ak, int ar, const double2 *Bs, int bk, int bc, int kb,
                                      int mrows, int ncols, Tile64<double2, true> &acc, int t) {
    const int w = t >> 5, lane = t & 31, g = lane >> 2;
    const int rb0 = w % 4, cb0 = 4 * (w / 4);
    if (8 * rb0 >= mrows || 8 * cb0 >= ncols) return;   // warp-uniform: none of this warp's blocks is used
    for (int k0 = 0; k0 < kb; k0 += 4) {
        const int kk = k0 + (lane & 3);
        const bool kin = kk < kb;
        double2 bf[4];
#pragma unroll
        for (int ci = 0; ci < 4; ++ci) {
            const int c = 8 * (cb0 + ci) + g;
            bf[ci] = kin && c < ncols ? Bs[(size_t)kk * bk + (size_t)c * bc] : czero<double2>();
        }
#pragma unroll
        for (int ri = 0; ri < 2; ++ri) {
            const int rb = rb0 + 4 * ri;
            if (8 * rb >= mrows) break;   // warp-uniform
            const int r = 8 * rb + g;
            double2 af = kin && r < mrows ? As[(size_t)kk * ak + (size_t)r * ar] : czero<double2>();
            if (NEG) af = make_double2(-af.x, -af.y);
#pragma unroll
            for (int ci = 0; ci < 4; ++ci) {
                if (8 * (cb0 + ci) >= ncols) break;   // warp-uniform
                double2 &d0 = acc.v[4 * ri + ci][0], &d1 = acc.v[4 * ri + ci][1];
                dmma_884(af.x, bf[ci].x, d0.x, d1.x);    // Re += Ar Br
                dmma_884(-af.y, bf[ci].y, d0.x, d1.x);   //     - Ai Bi
                dmma_884(af.x, bf[ci].y, d0.y, d1.y);    // Im += Ar Bi
                dmma_884(af.y, bf[ci].x, d0.y, d1.y);    //     + Ai Br
            }
        }
    }
}

template <class R>
__global__ void k_front_gather(FactorArgs<R> a, int lvl_first) {
    using C = cplx<R>;
    const int node = a.s.lvl_nodes[lvl_first + blockIdx.y];
    const int f = a.s.nfront[node];
    const int j = blockIdx.x * GATHER_COLS + (threadIdx.x >> 5);   // one warp per front column
    if (j >= f) return;   // warp-uniform (no barrier below)
    C *base = reinterpret_cast<C *>(a.front) + (size_t)blockIdx.z * a.s.front_total;
    C *F = base + a.s.front_off[node];
    const int *inv = a.s.inv + a.s.inv_off[node];
    const int c0 = a.s.child0[node], c1 = a.s.child1[node];
    const int b0 = c0 >= 0 ? inv[j] : -1;
    const int b1 = c1 >= 0 ? inv[f + j] : -1;
    const C *cb0 = nullptr, *cb1 = nullptr;
    int f0 = 0, f1 = 0;
    if (b0 >= 0) {
        const int s0 = a.s.npiv[c0]; f0 = a.s.nfront[c0];
        cb0 = base + a.s.front_off[c0] + s0 + (size_t)(s0 + b0) * f0;
    }
    if (b1 >= 0) {
        const int s1 = a.s.npiv[c1]; f1 = a.s.nfront[c1];
        cb1 = base + a.s.front_off[c1] + s1 + (size_t)(s1 + b1) * f1;
    }
    for (int i = threadIdx.x & 31; i < f; i += 32) {
        C v = czero<C>();
        if (cb0) { const int r = inv[i]; if (r >= 0) v = cadd(v, cb0[r]); }
        if (cb1) { const int r = inv[f + i]; if (r >= 0) v = cadd(v, cb1[r]); }
        F[i + (size_t)j * f] = v;
    }
}

template <class R>
__global__ void k_entry_scatter(FactorArgs<R> a, int64_t e0, int64_t cnt) {
    using C = cplx<R>;
    const int64_t e = e0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= e0 + cnt) return;
    C *F = reinterpret_cast<C *>(a.front) + (size_t)blockIdx.y * a.s.front_total;
    const double2 v = a.A[(size_t)blockIdx.y * 9 * a.s.n + a.ent_src[e]];
    C &d = F[a.ent_dst[e]];
    d = cadd(d, cconv<C>(v));
}

// Static pivoting: a pivot of magnitude below pivtol (or NaN) is replaced by
// itself scaled to magnitude pivtol (pivtol when it is zero) and counted.
// The test compares squares, so the common case takes no square root.
template <class R>
__device__ __forceinline__ cplx<R> static_pivot(cplx<R> piv, R pivtol, int &npert) {
    const R m2 = cabs2(piv), tol2 = pivtol * pivtol;
    const bool small = tol2 > R(0) ? !(m2 >= tol2) : !(sqrt(m2) >= pivtol);   // also catches NaN
    if (small) {
        const R mag = sqrt(m2);
        if (mag > R(0)) {
            const R sc = pivtol / mag;
            piv = mk(piv.x * sc, piv.y * sc);
        } else {
            piv = mk(pivtol, R(0));
        }
        ++npert;
    }
    return piv;
}

// LU of the kb x kb diagonal block at (k0, k0) of the front F (leading
// dimension f), with threshold row exchanges inside the block or without
// (below), a pivot that stays tiny replaced as static_pivot does; the
// inverses of its two triangles are written back in its place (all that
// the panel products and the substitution use): L^-1 in the strict lower
// part (unit diagonal implied), U^-1 in the upper part with the diagonal.
//
// The inverses are built during the elimination, one rank-1 step per pivot
// p over every entry outside the leading (p+1) x (p+1) block, with l = the
// scaled column p of L and u = row p of U over the pivot:
//   trailing   D(r, c) -= l_r D(p, c)             r, c > p
//   L^-1       X(r, c) -= l_r X(p, c)             r > p >= c   (X = I initially)
//   unit U^-1  Z(r, c) -= Z(r, p) D(p, c) / piv   r <= p < c   (Z = I initially)
// (X = L_p^-1 ... L_0^-1 and Z = M_0^-1 ... M_p^-1 for the elementary
// factors L = L_0 L_1 ... and unit U = ... M_1 M_0), and U^-1 = Z diag(1/piv).
// All three are T(r, c) -= (a_r / piv) b_c with a = column p and b = row p
// of D where they lie beyond p, of X / Z otherwise; X and Z share one array
// (strict lower / upper part).  The regions are disjoint and read only row
// and column p, so one barrier per pivot suffices.  Each thread owns the
// entries (t % NB, t / NB + 8 k), k < 4 (256 threads), updated without
// branches.  (With three barriers per pivot and the inverses as column
// recurrences afterwards the block took about twice as long; the chain is
// the serial part of every pivot step of the upper levels.)
//
// Without row exchanges (PIV false) thread 0 forms the next pivot from row
// and column p before the step and publishes its reciprocal.  With them,
// warp 0 picks pivot p after step p - 1 (a second barrier): the row r >= p
// of largest |D(r, p)| is exchanged with row p when |D(p, p)|^2 <
// pivtau2 |D(r, p)|^2 -- the whole row of D (its multipliers included) and
// the finished part of X (columns < p: X' = P X P for the exchange P);
// Z only holds finished rows < p.  The block's permutation goes to
// pivsrc[vars[k0 + q]] (q: pivot position, value: block row in equation
// order); columns right of the block are exchanged when the U panel is
// staged, columns left of it (earlier blocks' multipliers) stay in equation
// order -- the forward substitution gathers the block's rows at the same
// point of the elimination.  The CTA has DIAG_THREADS threads; sm is shared
// scratch of DIAG_SCRATCH complex values.
constexpr int DIAG_SCRATCH = 2 * NB * (NB + 1) + NB;
constexpr int DIAG_THREADS = 256;

template <class R, bool PIV>
__device__ void factor_diag_block(const FactorArgs<R> &a, cplx<R> *F, int f, int k0, int kb, cplx<R> *sm,
                                  unsigned char *src, const int *vars) {
    using C = cplx<R>;
    constexpr int NE = NB * NB / DIAG_THREADS;   // entries per thread
    auto D = reinterpret_cast<C (*)[NB + 1]>(sm);
    auto W = reinterpret_cast<C (*)[NB + 1]>(sm + NB * (NB + 1));   // X (strict lower) and Z (upper)
    C *rdiag = sm + 2 * NB * (NB + 1);
    __shared__ int rowof[NB];   // PIV: block row (equation order) at pivot position q
    const R pivtol = (R)(a.pivscale * __longlong_as_double((long long)*a.amax));
    int np = 0, nsw = 0;   // pivots this thread perturbed / exchanged
    const int r = threadIdx.x % NB, cb = threadIdx.x / NB;
    if (PIV && threadIdx.x < NB) rowof[threadIdx.x] = threadIdx.x;
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        const int c = cb + (DIAG_THREADS / NB) * e;
        if (r < kb && c < kb) {
            C v = F[(k0 + r) + (size_t)(k0 + c) * f];
            if (!PIV && r == 0 && c == 0) {
                v = static_pivot<R>(v, pivtol, np);
                rdiag[0] = crcp(v);
            }
            D[r][c] = v;
            W[r][c] = r == c ? mk(R(1), R(0)) : czero<C>();
        }
    }
    __syncthreads();
    for (int p = 0; p < kb; ++p) {
        if (PIV) {
            if (threadIdx.x < 32) {   // warp 0: pivot p
                const int lane = threadIdx.x;
                R m2 = lane >= p && lane < kb ? cabs2(D[lane][p]) : R(-1);
                int arg = lane;
#pragma unroll
                for (int o = 16; o; o >>= 1) {
                    const R om = __shfl_xor_sync(0xffffffffu, m2, o);
                    const int oa = __shfl_xor_sync(0xffffffffu, arg, o);
                    if (om > m2 || (om == m2 && oa < arg)) {
                        m2 = om;
                        arg = oa;
                    }
                }
                m2 = __shfl_sync(0xffffffffu, m2, 0);   // lane 0's result for all (NaN entries
                arg = __shfl_sync(0xffffffffu, arg, 0);  // could leave the lanes disagreeing)
                const bool swap = arg != p && cabs2(D[p][p]) < (R)a.pivtau2 * m2;   // warp-uniform
                if (swap) {
                    if (lane < kb) {
                        const C t = D[p][lane];
                        D[p][lane] = D[arg][lane];
                        D[arg][lane] = t;
                        if (lane < p) {
                            const C u = W[p][lane];
                            W[p][lane] = W[arg][lane];
                            W[arg][lane] = u;
                        }
                    }
                    if (lane == 0) {
                        const int t = rowof[p];
                        rowof[p] = rowof[arg];
                        rowof[arg] = t;
                        ++nsw;
                    }
                    __syncwarp();
                }
                if (lane == 0) rdiag[p] = crcp(static_pivot<R>(D[p][p], pivtol, np));
            }
            __syncthreads();
            if (p + 1 == kb) break;
        } else if (p + 1 == kb) {
            break;
        }
        const C rp = rdiag[p];
        if (!PIV && threadIdx.x == 0) {
            C v = D[p + 1][p + 1];
            cfms(v, cmul(D[p + 1][p], rp), D[p][p + 1]);
            v = static_pivot<R>(v, pivtol, np);
            rdiag[p + 1] = crcp(v);
        }
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const int c = cb + (DIAG_THREADS / NB) * e;
            if (r < kb && c < kb && (r > p || c > p) && (PIV || !(r == p + 1 && c == p + 1))) {
                const C av = r > p ? D[r][p] : W[r][p];
                const C bv = c > p ? D[p][c] : W[p][c];
                C &T = (r > p && c > p) ? D[r][c] : W[r][c];
                C v = T;
                cfms(v, cmul(av, rp), bv);
                T = v;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        const int c = cb + (DIAG_THREADS / NB) * e;
        if (r < kb && c < kb) F[(k0 + r) + (size_t)(k0 + c) * f] = r > c ? W[r][c] : cmul(W[r][c], rdiag[c]);
    }
    if (PIV && threadIdx.x < kb) src[vars[k0 + threadIdx.x]] = (unsigned char)rowof[threadIdx.x];
    if (np) atomicAdd(a.npert, (unsigned long long)np);
    if (PIV && nsw) atomicAdd(a.nswap, (unsigned long long)nsw);
}

// the diagonal block (k0, kb) of front `node` in matrix z, with row
// exchanges when piv (the level's fronts have more than NB pivots)
template <class R>
__device__ __forceinline__ void diag_block(const FactorArgs<R> &a, cplx<R> *F, int node, int z, int k0, int kb,
                                           cplx<R> *sm, bool piv) {
    const int f = a.s.nfront[node];
    if (piv) {
        factor_diag_block<R, true>(a, F, f, k0, kb, sm, a.pivsrc + (size_t)z * a.s.n, a.s.vars + a.s.var_off[node]);
    } else {
        factor_diag_block<R, false>(a, F, f, k0, kb, sm, nullptr, nullptr);
    }
}

// K3a: the first diagonal block of every front of the level (the later
// ones are factored by the first CTA of the preceding trailing update)
template <class R>
__global__ void __launch_bounds__(DIAG_THREADS) k_diag(FactorArgs<R> a, int lvl_first, int piv) {
    using C = cplx<R>;
    const int node = a.s.lvl_nodes[lvl_first + blockIdx.x];
    const int s = a.s.npiv[node];
    if (s <= 0) return;
    C *F = reinterpret_cast<C *>(a.front) + (size_t)blockIdx.y * a.s.front_total + a.s.front_off[node];
    extern __shared__ unsigned char smem_raw[];
    diag_block<R>(a, F, node, blockIdx.y, 0, min(NB, s), reinterpret_cast<C *>(smem_raw), piv != 0);
}

// K3b: the L and U panels of pivot block k0 as products with the inverted
// triangles of its (already factored) diagonal block: L21 = A21 U11^-1 and
// U12 = L11^-1 A12, one 64-row (L) or 64-column (U) slice per CTA, 256
// threads.  Both are formed with kb rows of output (the L slice as its
// transpose U11^-T A21^T), so all eight warps of the matrix-instruction
// tile layout hold work.  Each CTA reads and writes only its own slice;
// the diagonal block is read-only here.
template <class R>
__global__ void __launch_bounds__(256) k_panel_mm(FactorArgs<R> a, int lvl_first, int k0, int ntmax, int piv) {
    using C = cplx<R>;
    const int node = a.s.lvl_nodes[lvl_first + blockIdx.y];
    const int s = a.s.npiv[node];
    if (k0 >= s) return;
    const int f = a.s.nfront[node];
    const int kb = min(NB, s - k0);
    const int i0 = k0 + kb;
    const bool upper = blockIdx.x >= (unsigned)ntmax;
    const int x0 = i0 + (upper ? blockIdx.x - ntmax : blockIdx.x) * TILE;   // first row (L) / column (U)
    if (x0 >= f) return;
    const int nx = min(TILE, f - x0);
    C *F = reinterpret_cast<C *>(a.front) + (size_t)blockIdx.z * a.s.front_total + a.s.front_off[node];

    extern __shared__ unsigned char smem_raw[];
    C *Is = reinterpret_cast<C *>(smem_raw);   // [NB][TSTR]: Is[k * TSTR + r] = triangle-inverse factor (r, k)
    C *Ps = Is + NB * TSTR;                    // [NB][TSTR]: Ps[k * TSTR + x] = panel entry (k, x)
    const C *Dg = F + k0 + (size_t)k0 * f;    // the inverted diagonal block
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        const int r = t % NB, k = t / NB;      // Is(r, k): U^-T (r, k) = U^-1 (k, r), or L^-1 (r, k)
        if (r < kb && k < kb) {
            if (upper) {
                if (k < r) cp_async_elem(Is + k * TSTR + r, Dg + r + (size_t)k * f);
                else Is[k * TSTR + r] = k == r ? mk(R(1), R(0)) : czero<C>();
            } else {
                if (k <= r) cp_async_elem(Is + k * TSTR + r, Dg + k + (size_t)r * f);
                else Is[k * TSTR + r] = czero<C>();
            }
        }
    }
    __shared__ unsigned char rsrc[NB];   // U slice: block row of pivot position k (row exchanges)
    if (upper) {
        if (threadIdx.x < NB)
            rsrc[threadIdx.x] = piv && threadIdx.x < kb
                                    ? a.pivsrc[(size_t)blockIdx.z * a.s.n + a.s.vars[a.s.var_off[node] + k0 + threadIdx.x]]
                                    : (unsigned char)threadIdx.x;
        __syncthreads();
    }
    for (int t = threadIdx.x; t < NB * TILE; t += blockDim.x) {
        if (upper) {   // A12 columns: contiguous along the pivot index; rows in pivot order
            const int x = t / NB, k = t % NB;
            if (k < kb && x < nx) cp_async_elem(Ps + k * TSTR + x, F + (k0 + rsrc[k]) + (size_t)(x0 + x) * f);
        } else {       // A21 rows: contiguous along the row index
            const int x = t % TILE, k = t / TILE;
            if (k < kb && x < nx) cp_async_elem(Ps + k * TSTR + x, F + (x0 + x) + (size_t)(k0 + k) * f);
        }
    }
    staged_sync();
    Tile64<C, sizeof(R) == 8> acc;
    for_tile64(acc, threadIdx.x, [](int, int, C &v) { v = czero<C>(); });
    mma64<false>(Is, TSTR, 1, Ps, TSTR, 1, kb, kb, nx, acc, threadIdx.x);
    for_tile64(acc, threadIdx.x, [&](int k, int x, C &v) {
        if (k < kb && x < nx) {
            if (upper) F[(k0 + k) + (size_t)(x0 + x) * f] = v;
            else F[(x0 + x) + (size_t)(k0 + k) * f] = v;
        }
    });
}

// Trailing update C -= Lp * Up on one TILE x TILE tile; 256 threads, each
// owns a 4 x 4 complex sub-tile with rows tx + 16a and columns ty + 16b.
// Only the part of the trailing matrix that still belongs to pivot rows or
// pivot columns is updated here; the contribution block (rows and columns
// >= npiv) receives all pivot steps at once in one K = npiv GEMM at the end
// of the level (launch_cb_gemm).
static_assert(DIAG_THREADS == 256, "k_update's first CTA factors the next diagonal block");
template <class R>
__global__ void __launch_bounds__(256) k_update(FactorArgs<R> a, int lvl_first, int k0, int ntmax, int piv) {
    using C = cplx<R>;
    const int node = a.s.lvl_nodes[lvl_first + blockIdx.y];
    const int s = a.s.npiv[node];
    if (k0 >= s) return;
    const int f = a.s.nfront[node];
    const int kb = min(NB, s - k0);
    const int i0 = k0 + kb, m = f - i0;
    const int nt = (m + TILE - 1) / TILE;
    C *F = reinterpret_cast<C *>(a.front) + (size_t)blockIdx.z * a.s.front_total + a.s.front_off[node];
    const int ti = blockIdx.x / ntmax, tj = blockIdx.x % ntmax;
    if (ti >= nt || tj >= nt) return;
    if (i0 + ti * TILE >= s && i0 + tj * TILE >= s) return;   // tile inside the contribution block

    extern __shared__ unsigned char smem_raw[];
    C *Ls = reinterpret_cast<C *>(smem_raw);   // [NB][TSTR]: Ls[c * TSTR + r]
    C *Us = Ls + NB * TSTR;                    // [NB][TSTR]: Us[c * TSTR + col]
    const int r0 = i0 + ti * TILE, c0 = i0 + tj * TILE;
    // a tile whose columns all lie in the contribution block needs only its
    // pivot rows (and the other way round): the product is cut to them
    const int mrows = c0 >= s ? min(TILE, s - r0) : min(TILE, f - r0);
    const int ncols = r0 >= s ? min(TILE, s - c0) : min(TILE, f - c0);
    // asynchronous copies, all in flight at once; entries outside those rows
    // and columns or beyond kb are not staged (the product reads k < kb only
    // and treats rows / columns outside them as zero)
    for (int t = threadIdx.x; t < NB * TILE; t += blockDim.x) {
        const int r = t % TILE, c = t / TILE;
        if (c < kb && r < mrows) cp_async_elem(Ls + c * TSTR + r, F + (r0 + r) + (size_t)(k0 + c) * f);
        const int col = t / NB, cc = t % NB;   // U: contiguous along the pivot index
        if (cc < kb && col < ncols) cp_async_elem(Us + cc * TSTR + col, F + (k0 + cc) + (size_t)(c0 + col) * f);
    }
    // the tile's current values go into the accumulators while the staged
    // operands land (read after the products, their latency was exposed)
    Tile64<C, sizeof(R) == 8> acc;
    auto mine = [&](int rr, int cc) { return rr < mrows && cc < ncols && (r0 + rr < s || c0 + cc < s); };
    for_tile64(acc, threadIdx.x, [&](int rr, int cc, C &v) {
        v = mine(rr, cc) ? F[(r0 + rr) + (size_t)(c0 + cc) * f] : czero<C>();
    });
    staged_sync();
    mma64<true>(Ls, TSTR, 1, Us, TSTR, 1, kb, mrows, ncols, acc, threadIdx.x);
    for_tile64(acc, threadIdx.x, [&](int rr, int cc, C &v) {
        if (mine(rr, cc)) F[(r0 + rr) + (size_t)(c0 + cc) * f] = v;
    });
    if (blockIdx.x == 0) {
        // the first tile holds the next diagonal block, now final: factor it
        // here (the first CTA starts first, so this overlaps the other tiles)
        __syncthreads();   // the tile's global writes are visible; Ls / Us are free
        diag_block<R>(a, F, node, blockIdx.z, i0, min(NB, s - i0), Ls, piv != 0);
    }
}

// Batched C -= A * B on CUDA cores (64 x 64 output tiles, 4 x 4 complex
// register tile per thread): the contribution-block update of every front
// of a level in one launch.  K runs in chunks of GKC staged through shared
// memory by asynchronous copies, two buffers: the next chunk's loads are in
// flight while the current one is multiplied.  Tile entries outside A's
// rows or B's columns are not staged (they only feed accumulators that are
// never stored); the chunk loop reads only the k < kb part.
constexpr int GKC = 16;

template <class R>
__global__ void __launch_bounds__(256) k_gemm_sub_cc(const GemmProb<R> *__restrict__ probs,
                                                     const int4 *__restrict__ tiles) {
    using C = cplx<R>;
    const int4 tl = tiles[blockIdx.x];
    const GemmProb<R> p = probs[tl.x];
    const int r0 = tl.y * TILE, c0 = tl.z * TILE;
    extern __shared__ unsigned char smem_raw[];
    C *As = reinterpret_cast<C *>(smem_raw);   // [2][GKC][TSTR]: As[c * TSTR + r]
    C *Bs = As + 2 * GKC * TSTR;               // [2][GKC][TSTR]: Bs[c * TSTR + col]
    auto stage = [&](int buf, int k0) {
        const int kb = min(GKC, p.k - k0);
        C *Ab = As + buf * GKC * TSTR, *Bb = Bs + buf * GKC * TSTR;
        for (int t = threadIdx.x; t < GKC * TILE; t += blockDim.x) {
            const int r = t % TILE, c = t / TILE;
            if (c < kb && r0 + r < p.m) cp_async_elem(Ab + c * TSTR + r, p.A + (size_t)(r0 + r) + (size_t)(k0 + c) * p.lda);
            const int col = t / GKC, cc = t % GKC;   // B: contiguous along k
            if (cc < kb && c0 + col < p.n)
                cp_async_elem(Bb + cc * TSTR + col, p.B + (size_t)(k0 + cc) + (size_t)(c0 + col) * p.ldb);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    Tile64<C, sizeof(R) == 8> acc;
    for_tile64(acc, threadIdx.x, [](int, int, C &v) { v = czero<C>(); });
    const int mrows = min(TILE, p.m - r0), ncols = min(TILE, p.n - c0);
    const int nk = (p.k + GKC - 1) / GKC;
    if (nk > 0) stage(0, 0);
    for (int kc = 0; kc < nk; ++kc) {
        if (kc + 1 < nk) {
            stage((kc + 1) & 1, (kc + 1) * GKC);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");   // chunk kc has landed
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
        const int kb = min(GKC, p.k - kc * GKC);
        mma64<false>(As + (kc & 1) * GKC * TSTR, TSTR, 1, Bs + (kc & 1) * GKC * TSTR, TSTR, 1, kb, mrows, ncols, acc,
                     threadIdx.x);
        __syncthreads();   // this buffer is staged again for chunk kc + 2
    }
    for_tile64(acc, threadIdx.x, [&](int rr, int cc, C &v) {
        const int row = r0 + rr, col = c0 + cc;
        if (row < p.m && col < p.n) {
            C &d = p.C[(size_t)row + (size_t)col * p.ldc];
            d = csub(d, v);
        }
    });
}

template <class R>
void launch_gemm_sub_cc(const GemmProb<R> *d_probs, const int4 *d_tiles, int ntiles, cudaStream_t st) {
    if (ntiles <= 0) return;
    const size_t smem = 4 * GKC * TSTR * sizeof(cplx<R>);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gemm_sub_cc<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    (k_gemm_sub_cc<R><<<ntiles, 256, smem, st>>>(d_probs, d_tiles), note_launch());
}

template void launch_gemm_sub_cc<double>(const GemmProb<double> *, const int4 *, int, cudaStream_t);
template void launch_gemm_sub_cc<float>(const GemmProb<float> *, const int4 *, int, cudaStream_t);

template <class R>
void launch_factor_level(const FactorArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    using C = cplx<R>;
    if (L.count == 0) return;
    for_level_pieces(L, [&](int first, int count) {
        (k_front_gather<R><<<dim3((L.max_front + GATHER_COLS - 1) / GATHER_COLS, count, a.nf), 32 * GATHER_COLS, 0,
                             st>>>(a, first),
         note_launch());
    });
    if (L.ent_count > 0) {
        const int tpb = 256;
        (k_entry_scatter<R><<<dim3((unsigned)((L.ent_count + tpb - 1) / tpb), a.nf), tpb, 0, st>>>(a, L.ent_first,
                                                                                                  L.ent_count), note_launch());
    }
    const size_t smem = 2 * NB * TSTR * sizeof(C);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_update<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_panel_mm<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set = true;
    }
    const int piv = a.pivsrc && a.pivtau2 > 0;   // row exchanges (every level of this route)
    for_level_pieces(L, [&](int first, int count) {
        (k_diag<R><<<dim3(count, a.nf), DIAG_THREADS, DIAG_SCRATCH * sizeof(C), st>>>(a, first, piv), note_launch());
    });
    for (int k0 = 0; k0 < L.max_piv; k0 += NB) {
        const int mmax = L.max_front - k0 - 1;   // largest trailing size (kb >= 1)
        const int ntmax = mmax > 0 ? (mmax + TILE - 1) / TILE : 0;
        if (ntmax > 0)
            for_level_pieces(L, [&](int first, int count) {
                (k_panel_mm<R><<<dim3(2 * ntmax, count, a.nf), 256, smem, st>>>(a, first, k0, ntmax, piv), note_launch());
            });
        // the trailing tiles only update pivot rows and columns still to
        // come (and factor the next diagonal block): after the level's last
        // pivot block there is nothing left for them
        if (ntmax > 0 && L.max_piv > k0 + NB)
            for_level_pieces(L, [&](int first, int count) {
                (k_update<R><<<dim3(ntmax * ntmax, count, a.nf), 256, smem, st>>>(a, first, k0, ntmax, piv),
                 note_launch());
            });
    }
}

template void launch_factor_level<double>(const FactorArgs<double> &, const LevelInfo &, cudaStream_t);
template void launch_factor_level<float>(const FactorArgs<float> &, const LevelInfo &, cudaStream_t);

// ---------------------------------------------------------------------
// Small fronts (the lower levels of the tree): one CTA assembles and
// factorises a whole front in shared memory -- extend-add of the children's
// contribution blocks, the operator entries, right-looking LU of the npiv
// pivot columns with the same static pivoting as factor_diag_block, the Schur
// complement of the contribution block, and the inverses of the NB x NB
// diagonal blocks -- and writes the front back once.  The result has the
// layout the blocked path leaves (L below, U above, diagonal-block inverses,
// contribution block), in one launch per level instead of the
// gather / scatter / ceil(npiv/NB) x (panel + update) / contribution GEMM
// sequence.  S[i + j * ld] holds front entry (i, j).
// ---------------------------------------------------------------------
constexpr int SMALL_FT = 256;   // threads per CTA

// (register bounds: three CTAs per SM for the blocked form, whose panel
// registers would otherwise cost one; four for the per-pivot form, which the
// smaller fronts of levels 1-2 fit in shared memory -- without a bound the
// compiler takes 88 registers and two CTAs, and those levels run 2x slower)
template <class R, int SROWS, bool BLOCKED>
__global__ void __launch_bounds__(SMALL_FT, BLOCKED ? 3 : 4) k_factor_small(FactorArgs<R> a, int lvl_first, int ld) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    __shared__ C Dinv[NB][NB + 1];
    __shared__ int npert;
    const int pos = lvl_first + blockIdx.x;
    const int node = a.s.lvl_nodes[pos];
    const int f = a.s.nfront[node], s = a.s.npiv[node];
    C *rd = S + (size_t)ld * f;   // reciprocal pivots
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = SMALL_FT / 32;
    const size_t fz = blockIdx.y;
    C *base = reinterpret_cast<C *>(a.front) + fz * a.s.front_total;
    C *F = base + a.s.front_off[node];

    // extend-add of the children's contribution blocks (zero for leaves)
    const int *inv = a.s.inv + a.s.inv_off[node];
    const int c0 = a.s.child0[node], c1 = a.s.child1[node];
    const C *cb0 = nullptr, *cb1 = nullptr;
    int f0 = 0, f1 = 0;
    if (c0 >= 0) { const int s0 = a.s.npiv[c0]; f0 = a.s.nfront[c0]; cb0 = base + a.s.front_off[c0] + s0 + (size_t)s0 * f0; }
    if (c1 >= 0) { const int s1 = a.s.npiv[c1]; f1 = a.s.nfront[c1]; cb1 = base + a.s.front_off[c1] + s1 + (size_t)s1 * f1; }
    for (int j = warp; j < f; j += nw) {
        const int j0 = cb0 ? inv[j] : -1, j1 = cb1 ? inv[f + j] : -1;
        for (int i = lane; i < f; i += 32) {
            C v = czero<C>();
            if (j0 >= 0) { const int r = inv[i]; if (r >= 0) v = cadd(v, cb0[r + (size_t)j0 * f0]); }
            if (j1 >= 0) { const int r = inv[f + i]; if (r >= 0) v = cadd(v, cb1[r + (size_t)j1 * f1]); }
            S[i + j * ld] = v;
        }
    }
    if (tid == 0) npert = 0;
    __syncthreads();
    // operator entries owned by the front (positions are distinct)
    {
        const int64_t e0 = a.ent_lvl_off[pos], e1 = a.ent_lvl_off[pos + 1];
        const int64_t fo = a.s.front_off[node];
        const double2 *A = a.A + fz * 9 * (size_t)a.s.n;
        for (int64_t e = e0 + tid; e < e1; e += SMALL_FT) {
            const int p = (int)(a.ent_dst[e] - fo);
            const int i = p % f, j = p / f;
            C &d = S[i + j * ld];
            d = cadd(d, cconv<C>(A[a.ent_src[e]]));
        }
    }
    __syncthreads();

    // right-looking LU of the pivot columns; the trailing update covers the
    // contribution block too (its Schur complement).  Warp 0 updates column
    // k + 1 first in step k, so it can take the next pivot (static pivoting
    // as in factor_diag_block) and scale the next L column while the other warps are
    // still updating: one barrier per pivot.
    const R pivtol = (R)(a.pivscale * __longlong_as_double((long long)*a.amax));
    auto take_pivot = [&](int k) {   // warp 0 only: pivot k, reciprocal, L column k scaled
        if (lane == 0) {
            const C piv = static_pivot<R>(S[k + k * ld], pivtol, npert);
            S[k + k * ld] = piv;
            rd[k] = crcp(piv);
        }
        __syncwarp();
        const C rk = rd[k];
        for (int i = k + 1 + lane; i < f; i += 32) S[i + k * ld] = cmul(S[i + k * ld], rk);
        __syncwarp();
    };
    if constexpr (BLOCKED) {
        // complex128, fronts with many pivots: blocked by 4-pivot panels.  Warp 0 factors a panel's
        // columns (static pivoting, L columns scaled) and applies each pivot
        // to the panel rows right of the panel (the U rows); then every warp
        // applies the rank-4 update to the trailing block on FP64 matrix
        // instructions, one 8 x 8 block per warp at a time.  Two barriers per
        // panel instead of one per pivot.
        constexpr int PW = 4;
        const int g = lane >> 2, kq = lane & 3;
        for (int kb0 = 0; kb0 < s; kb0 += PW) {
            const int kend = min(s, kb0 + PW);
            if (warp == 0) {
                // the panel in registers: lane l holds rows l and l + 32
                // (fronts of at most 64 rows) of the panel's columns; the
                // pivot row's entries come from their owner by shuffles, so
                // each pivot costs shuffles and FMAs, no shared-memory round
                // trip or warp barrier
                C pv[2][PW];
#pragma unroll
                for (int q = 0; q < 2; ++q)
#pragma unroll
                    for (int j = 0; j < PW; ++j) {
                        const int i = lane + 32 * q;
                        pv[q][j] = i < f && kb0 + j < kend ? S[i + (kb0 + j) * ld] : czero<C>();
                    }
#pragma unroll
                for (int jk = 0; jk < PW; ++jk) {
                    const int k = kb0 + jk;
                    if (k >= kend) break;   // warp-uniform
                    const int owner = k & 31;
                    C prow[PW];   // row k of the panel
#pragma unroll
                    for (int j = 0; j < PW; ++j) {
                        const C v = k >= 32 ? pv[1][j] : pv[0][j];
                        prow[j] = make_double2(__shfl_sync(0xffffffffu, v.x, owner), __shfl_sync(0xffffffffu, v.y, owner));
                    }
                    int np = 0;
                    const C piv = static_pivot<R>(prow[jk], pivtol, np);   // every lane: the same pivot
                    const C rk = crcp(piv);
                    if (lane == 0) {
                        rd[k] = rk;
                        npert += np;
                    }
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const int i = lane + 32 * q;
                        if (i == k) pv[q][jk] = piv;   // the (perturbed) pivot
                        if (i > k && i < f) {
                            const C l = cmul(pv[q][jk], rk);
                            pv[q][jk] = l;
#pragma unroll
                            for (int j = jk + 1; j < PW; ++j) cfms(pv[q][j], l, prow[j]);
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < 2; ++q)
#pragma unroll
                    for (int j = 0; j < PW; ++j) {
                        const int i = lane + 32 * q;
                        if (i < f && kb0 + j < kend) S[i + (kb0 + j) * ld] = pv[q][j];
                    }
                __syncwarp();
                // the panel's U rows right of the panel: unit lower solve with
                // the panel's diagonal block, one column per lane
                const int pw = kend - kb0;
                for (int j = kend + lane; j < f; j += 32) {
                    C u[PW];
#pragma unroll
                    for (int r = 0; r < PW; ++r) {
                        if (r >= pw) break;
                        C v = S[kb0 + r + j * ld];
#pragma unroll
                        for (int t = 0; t < r; ++t) cfms(v, S[kb0 + r + (kb0 + t) * ld], u[t]);
                        u[r] = v;
                        S[kb0 + r + j * ld] = v;
                    }
                }
            }
            __syncthreads();
            const int mt = f - kend, nbt = (mt + 7) / 8;
            for (int bi = warp; bi < nbt * nbt; bi += nw) {   // trailing block -= L(:, panel) U(panel, :)
                const int r = kend + 8 * (bi % nbt) + g, c0 = kend + 8 * (bi / nbt);
                const int cl = c0 + 2 * kq;
                double2 d0 = r < f && cl < f ? S[r + cl * ld] : czero<C>();
                double2 d1 = r < f && cl + 1 < f ? S[r + (cl + 1) * ld] : czero<C>();
                const int kk = kb0 + kq;
                const bool kin = kk < kend;
                double2 af = kin && r < f ? S[r + kk * ld] : czero<C>();
                af = make_double2(-af.x, -af.y);
                const int cb = c0 + g;
                const double2 bf = kin && cb < f ? S[kk + cb * ld] : czero<C>();
                dmma_884(af.x, bf.x, d0.x, d1.x);
                dmma_884(-af.y, bf.y, d0.x, d1.x);
                dmma_884(af.x, bf.y, d0.y, d1.y);
                dmma_884(af.y, bf.x, d0.y, d1.y);
                if (r < f && cl < f) S[r + cl * ld] = d0;
                if (r < f && cl + 1 < f) S[r + (cl + 1) * ld] = d1;
            }
            __syncthreads();
        }
    } else {
        if (warp == 0 && s > 0) take_pivot(0);
        __syncthreads();
        // Each lane holds its rows of the scaled L column k in registers for the
        // whole step (SROWS x 32 >= the level's largest front), so an entry's
        // update reads shared memory once, not twice.
        for (int k = 0; k < s; ++k) {
            const int m = f - k - 1;
            C lk[SROWS];
#pragma unroll
            for (int q = 0; q < SROWS; ++q) {
                const int ii = lane + 32 * q;
                lk[q] = ii < m ? S[k + 1 + ii + k * ld] : czero<C>();
            }
            for (int jj = warp; jj < m; jj += nw) {
                C *col = S + (k + 1 + jj) * ld;
                const C u = col[k];
#pragma unroll
                for (int q = 0; q < SROWS; ++q) {
                    const int ii = lane + 32 * q;
                    if (ii < m) cfms(col[k + 1 + ii], lk[q], u);
                }
                if (jj == 0 && k + 1 < s) {   // warp 0 just finished column k + 1
                    __syncwarp();
                    take_pivot(k + 1);
                }
            }
            __syncthreads();
        }
    }

    // inverses of the NB x NB diagonal blocks: L^-1 strictly below the
    // diagonal (unit diagonal implied), U^-1 on and above it
    for (int k0 = 0; k0 < s; k0 += NB) {
        const int kb = min(NB, s - k0);
        auto D = [&](int r, int q) { return S[(k0 + r) + (k0 + q) * ld]; };
        if (tid < kb) {
            const int c = tid;
            for (int r = c + 1; r < kb; ++r) {
                C acc = D(r, c);
                for (int q = c + 1; q < r; ++q) cfma(acc, D(r, q), Dinv[q][c]);
                Dinv[r][c] = mk(-acc.x, -acc.y);
            }
        } else if (tid >= 32 && tid < 32 + kb) {
            const int c = tid - 32;
            Dinv[c][c] = rd[k0 + c];
            for (int r = c - 1; r >= 0; --r) {
                C acc = czero<C>();
                for (int q = r + 1; q <= c; ++q) cfma(acc, D(r, q), Dinv[q][c]);
                Dinv[r][c] = cmul(mk(-acc.x, -acc.y), rd[k0 + r]);
            }
        }
        __syncthreads();
        for (int t = tid; t < kb * kb; t += SMALL_FT) {
            const int r = t % kb, c = t / kb;
            S[(k0 + r) + (k0 + c) * ld] = Dinv[r][c];
        }
        __syncthreads();
    }

    for (int j = warp; j < f; j += nw)
        for (int i = lane; i < f; i += 32) F[i + (size_t)j * f] = S[i + j * ld];
    if (tid == 0 && npert) atomicAdd(a.npert, (unsigned long long)npert);
}

constexpr size_t SMALL_FACTOR_SMEM = 100 << 10;

template <class R>
static size_t small_factor_smem(int fmax) {
    const int ld = fmax + 1;
    return ((size_t)ld * fmax + fmax) * sizeof(cplx<R>);
}

template <class R>
bool small_factor_level(const LevelInfo &L) {   // (the shared-memory bound keeps fronts below 4 x 32 rows)
    return L.count > 0 && L.max_front <= 128 && small_factor_smem<R>(L.max_front) <= SMALL_FACTOR_SMEM;
}

template <class R>
void launch_factor_small(const FactorArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_factor_small<R, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMALL_FACTOR_SMEM);
        cudaFuncSetAttribute(k_factor_small<R, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMALL_FACTOR_SMEM);
        cudaFuncSetAttribute(k_factor_small<R, 4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMALL_FACTOR_SMEM);
        if (sizeof(R) == 8)
            cudaFuncSetAttribute(k_factor_small<R, 2, sizeof(R) == 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMALL_FACTOR_SMEM);
        attr_set = true;
    }
    const size_t smem = small_factor_smem<R>(L.max_front);
    const dim3 grid(L.count, a.nf);
    const int ld = L.max_front + 1;
    // the blocked complex128 LU pays on fronts with many pivots (the leaf
    // level: 5.4 -> 4.6 ms); with 7-13 pivots its one-warp panels are slower
    // GM_BLOCKED_LU_MIN_PIV=<n> moves the threshold (a large n: the
    // per-pivot kernel everywhere)
    static const int min_piv = [] {
        const char *v = std::getenv("GM_BLOCKED_LU_MIN_PIV");
        return v ? std::atoi(v) : 16;
    }();
    if (sizeof(R) == 8 && L.max_piv >= min_piv && L.max_front <= 64)   // (the blocked panel holds 64 rows)
        (k_factor_small<R, 2, sizeof(R) == 8><<<grid, SMALL_FT, smem, st>>>(a, L.first, ld), note_launch());
    else if (L.max_front <= 64) (k_factor_small<R, 2, false><<<grid, SMALL_FT, smem, st>>>(a, L.first, ld), note_launch());
    else if (L.max_front <= 96) (k_factor_small<R, 3, false><<<grid, SMALL_FT, smem, st>>>(a, L.first, ld), note_launch());
    else (k_factor_small<R, 4, false><<<grid, SMALL_FT, smem, st>>>(a, L.first, ld), note_launch());
}

template bool small_factor_level<double>(const LevelInfo &);
template bool small_factor_level<float>(const LevelInfo &);
template void launch_factor_small<double>(const FactorArgs<double> &, const LevelInfo &, cudaStream_t);
template void launch_factor_small<float>(const FactorArgs<float> &, const LevelInfo &, cudaStream_t);

// Grid-stride max of |A| with one atomicMax per warp.  Non-negative doubles
// order like their bit patterns read as unsigned integers.
__global__ void __launch_bounds__(256) k_amax(const double2 *A, size_t cnt, unsigned long long *out) {
    double m = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x) {
        const double2 v = A[i];
        const double a = hypot(v.x, v.y);
        m = (a > m || a != a) ? a : m;   // a NaN entry makes the maximum NaN (reported by the host)
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double q = __shfl_xor_sync(0xffffffffu, m, o);
        m = (q > m || q != q) ? q : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

void launch_amax(const double2 *A, size_t cnt, unsigned long long *out, cudaStream_t st) {
    note_launch();
    k_amax<<<148 * 8, 256, 0, st>>>(A, cnt, out);
}

__global__ void k_pack_split(double2 *dst, const double *re, const double *im, size_t cnt) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = make_double2(re[i], im[i]);
}

void launch_pack_split(double2 *dst, const double *re, const double *im, size_t cnt, cudaStream_t st) {
    note_launch();
    k_pack_split<<<148 * 8, 256, 0, st>>>(dst, re, im, cnt);
}

}  // namespace gm


namespace gm {

// ---------------------------------------------------------------------
// Mid-level fronts: at most NB pivots and at most MID_FT rows, but too
// large for the small kernel's whole-front tile.  After the extend-add
// gather and the operator entries (K2), one CTA per front and frequency
//   1. factorises the pivot columns (f x s) right-looking with each thread
//      holding one front row in registers: per pivot, warp 0 picks the
//      pivot row by the threshold rule (mid_select_pivot: rows keep their
//      threads and trade pivot positions), and the row's owner replaces a
//      pivot that stays tiny as static_pivot does and publishes the row and
//      the pivot's reciprocal in shared memory: one barrier per pivot, and
//      no shared-memory traffic for the update itself;
//   2. solves L11 U12 = P A12 with each thread holding one column of U12;
//   3. inverts the pivot block's two triangles;
//   4. writes L, U and the inverses back (the layout the blocked path
//      leaves);
//   5. applies the rank-s Schur update to the contribution block,
//      64 x 64 tiles of 4 x 4 complex per thread, each tile's old values
//      loaded into the accumulators first.
// This replaces the K3 / K4 steps and the level's contribution GEMM.
// Shared memory: P[i + c * (f + 1)] the pivot columns, then
// U[r + j * (s | 1)] the U12 rows (odd strides: conflict-free 16-byte
// accesses).
// ---------------------------------------------------------------------
constexpr int MID_FT = 256;   // threads per CTA, also the largest front handled

// Warp 0 of k_factor_mid (which holds every pivot row): pivot position kp
// goes to the row of largest |x[kp]| among the rows at positions >= kp when
// the row there has |x[kp]|^2 < tau2 times that (c2: this lane's
// |x[kp]|^2, pos: the pivot position of this lane's row; the two rows swap
// positions).  Only scalars: the caller's row stays in registers.
template <class R>
__device__ __forceinline__ void mid_select_pivot(R c2, int &pos, int kp, int s, R tau2, int &nsw) {
    const int lane = threadIdx.x & 31;
    R m2 = pos >= kp && pos < s ? c2 : R(-1);
    int arg = lane;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const R om = __shfl_xor_sync(0xffffffffu, m2, o);
        const int oa = __shfl_xor_sync(0xffffffffu, arg, o);
        if (om > m2 || (om == m2 && oa < arg)) {
            m2 = om;
            arg = oa;
        }
    }
    m2 = __shfl_sync(0xffffffffu, m2, 0);     // lane 0's result for all (NaN entries
    arg = __shfl_sync(0xffffffffu, arg, 0);   // could leave the lanes disagreeing)
    const int cur = __ffs(__ballot_sync(0xffffffffu, pos == kp)) - 1;   // the lane at position kp
    const R d2 = __shfl_sync(0xffffffffu, c2, cur);
    if (arg != cur && d2 < tau2 * m2) {   // warp-uniform
        const int pa = __shfl_sync(0xffffffffu, pos, arg);
        if (lane == cur) pos = pa;
        if (lane == arg) pos = kp;
        ++nsw;
    }
}

template <class R, int NPR>
__global__ void __launch_bounds__(MID_FT) k_factor_mid(FactorArgs<R> a, int lvl_first) {
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ C Dinv[NB][NB + 1];
    __shared__ C urow[2][NPR];   // pivot row k at columns k .. s-1, alternating buffers
    __shared__ C rd[NPR];        // reciprocal pivots
    __shared__ int perm[NB];     // front row at pivot position q (row exchanges)
    __shared__ int npert;
    const int node = a.s.lvl_nodes[lvl_first + blockIdx.x];
    const int f = a.s.nfront[node], s = a.s.npiv[node], m = f - s;
    if (s == 0) return;   // the gathered front is already the contribution block
    const int ldp = f + 1, ldu = s | 1;
    C *P = reinterpret_cast<C *>(smem_raw);
    C *U = P + (size_t)ldp * s;
    const int tid = threadIdx.x;
    C *F = reinterpret_cast<C *>(a.front) + (size_t)blockIdx.y * a.s.front_total + a.s.front_off[node];
    const R pivtol = (R)(a.pivscale * __longlong_as_double((long long)*a.amax));
    if (tid == 0) npert = 0;

    for (int t = tid; t < s * m; t += MID_FT) {   // A12, down each column, landing during step 1
        const int j = t / s, r = t - j * s;
        cp_async_elem(U + r + j * ldu, F + r + (size_t)(s + j) * f);
    }

    // 1. pivot columns, one row per thread.  Iteration k applies pivot k
    // and publishes pivot k + 1: the row at pivot position k + 1 and the
    // reciprocal.  Rows stay with their threads; pos is the pivot position
    // of the thread's row (its own index but for exchanged pivot rows).
    // With row exchanges (piv), warp 0 -- which holds every pivot row,
    // s <= 32 -- first gives position k + 1 to the row r of largest
    // |x_r[k+1]| among those at positions > k when the row there has
    // |x[k+1]|^2 < pivtau2 |x_r[k+1]|^2 (the two rows swap positions); the
    // rows go to shared memory at their positions afterwards.
    const bool own = tid < f;
    const bool piv = a.pivsrc != nullptr && a.pivtau2 > 0;
    C x[NPR];
#pragma unroll
    for (int j = 0; j < NPR; ++j) x[j] = (own && j < s) ? F[tid + (size_t)j * f] : czero<C>();
    int np = 0, nsw = 0, pos = tid;
    if (piv && tid < 32) mid_select_pivot<R>(cabs2(x[0]), pos, 0, s, (R)a.pivtau2, nsw);
    if (pos == 0) {
        x[0] = static_pivot<R>(x[0], pivtol, np);
        rd[0] = crcp(x[0]);
#pragma unroll
        for (int j = 0; j < NPR; ++j)
            if (j < s) urow[0][j] = x[j];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NPR; ++k) {
        if (k >= s) continue;   // s is the same for the whole CTA
        if (own && pos > k) {
            const C l = cmul(x[k], rd[k]);
            x[k] = l;
#pragma unroll
            for (int j = k + 1; j < NPR; ++j)
                if (j < s) cfms(x[j], l, urow[k & 1][j]);
        }
        const int k1 = k + 1 < NPR ? k + 1 : NPR - 1;   // pivot published by this iteration
        if (k + 1 < NPR && k + 1 < s) {
            if (piv && tid < 32) mid_select_pivot<R>(cabs2(x[k1]), pos, k1, s, (R)a.pivtau2, nsw);
            if (pos == k1 && own) {   // the row at the next pivot position
                x[k1] = static_pivot<R>(x[k1], pivtol, np);
                rd[k1] = crcp(x[k1]);
#pragma unroll
                for (int j = k1; j < NPR; ++j)
                    if (j < s) urow[k1 & 1][j] = x[j];
            }
        }
        __syncthreads();
    }
    if (own) {
#pragma unroll
        for (int j = 0; j < NPR; ++j)
            if (j < s) P[pos + j * ldp] = x[j];
        if (pos < s) perm[pos] = tid;
    }
    if (np) atomicAdd(&npert, np);
    if (tid == 0 && nsw) atomicAdd(a.nswap, (unsigned long long)nsw);
    staged_sync();
    if (piv && tid < s) a.pivsrc[(size_t)blockIdx.y * a.s.n + a.s.vars[a.s.var_off[node] + tid]] = (unsigned char)perm[tid];

    // 2. U12 = L11^-1 A12, one column per thread of warps 2 .. 7, while
    // warps 0 and 1 invert the pivot block's triangles (3.)
    for (int j = tid - 64; j >= 0 && j < m; j += MID_FT - 64) {
        C u[NPR];   // A12's rows in pivot order
#pragma unroll
        for (int r = 0; r < NPR; ++r) u[r] = r < s ? U[(piv ? perm[r] : r) + j * ldu] : czero<C>();
#pragma unroll
        for (int k = 0; k + 1 < NPR; ++k) {
            if (k + 1 < s) {
                const C uk = u[k];
#pragma unroll
                for (int r = k + 1; r < NPR; ++r)
                    if (r < s) cfms(u[r], P[r + k * ldp], uk);
            }
        }
#pragma unroll
        for (int r = 0; r < NPR; ++r)
            if (r < s) U[r + j * ldu] = u[r];
    }

    // 3. inverses of the pivot block's triangles: L^-1 strictly below the
    // diagonal (unit diagonal implied), U^-1 on and above it
    if (tid < s) {
        const int c = tid;
        for (int r = c + 1; r < s; ++r) {
            C acc = P[r + c * ldp];
            for (int q = c + 1; q < r; ++q) cfma(acc, P[r + q * ldp], Dinv[q][c]);
            Dinv[r][c] = mk(-acc.x, -acc.y);
        }
    } else if (tid >= 32 && tid < 32 + s) {
        const int c = tid - 32;
        Dinv[c][c] = rd[c];
        for (int r = c - 1; r >= 0; --r) {
            C acc = czero<C>();
            for (int q = r + 1; q <= c; ++q) cfma(acc, P[r + q * ldp], Dinv[q][c]);
            Dinv[r][c] = cmul(mk(-acc.x, -acc.y), rd[r]);
        }
    }
    __syncthreads();

    // 4. write back: pivot columns (inverses in the pivot block), U12
    for (int t = tid; t < f * s; t += MID_FT) {
        const int c = t / f, i = t - c * f;
        F[t] = i < s ? Dinv[i][c] : P[i + c * ldp];
    }
    for (int t = tid; t < s * m; t += MID_FT) {
        const int j = t / s, r = t - j * s;
        F[r + (size_t)(s + j) * f] = U[r + j * ldu];
    }
    if (tid == 0 && npert) atomicAdd(a.npert, (unsigned long long)npert);

    // 5. contribution block -= L21 U12, 64 x 64 tiles, each tile's old
    // values loaded into the accumulators first
    for (int i0 = 0; i0 < m; i0 += 64)
        for (int j0 = 0; j0 < m; j0 += 64) {
            Tile64<C, (sizeof(R) == 8 && NPR > 16)> acc;   // short K (<= 16 pivots): CUDA-core FMAs
            for_tile64(acc, tid, [&](int rr, int cc, C &v) {
                const int i = i0 + rr, j = j0 + cc;
                v = (i < m && j < m) ? F[s + i + (size_t)(s + j) * f] : czero<C>();
            });
            mma64<true>(P + s + i0, ldp, 1, U + (size_t)j0 * ldu, 1, ldu, s, min(64, m - i0), min(64, m - j0), acc,
                        tid);
            for_tile64(acc, tid, [&](int rr, int cc, C &v) {
                const int i = i0 + rr, j = j0 + cc;
                if (i < m && j < m) F[s + i + (size_t)(s + j) * f] = v;
            });
        }
}

constexpr size_t MID_FACTOR_SMEM = 200 << 10;

template <class R>
bool mid_factor_level(const LevelInfo &L) {
    return L.count > 0 && L.max_piv <= NB && L.max_front <= MID_FT && !small_factor_level<R>(L) &&
           (size_t)L.mid_words * sizeof(cplx<R>) <= MID_FACTOR_SMEM;
}

// Row exchanges happen on every level but those of the small-front kernel
// (whose fronts fit shared memory whole: the lower levels)
template <class R>
bool level_pivots(const LevelInfo &L) {
    return L.count > 0 && !small_factor_level<R>(L);
}
template bool level_pivots<double>(const LevelInfo &);
template bool level_pivots<float>(const LevelInfo &);

template <class R, int NPR>
static void launch_mid(const FactorArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_factor_mid<R, NPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MID_FACTOR_SMEM);
        attr_set = true;
    }
    (k_factor_mid<R, NPR><<<dim3(L.count, a.nf), MID_FT, (size_t)L.mid_words * sizeof(cplx<R>), st>>>(a, L.first),
     note_launch());
}

template <class R>
void launch_factor_mid(const FactorArgs<R> &a, const LevelInfo &L, cudaStream_t st) {
    for_level_pieces(L, [&](int first, int count) {
        (k_front_gather<R><<<dim3((L.max_front + GATHER_COLS - 1) / GATHER_COLS, count, a.nf), 32 * GATHER_COLS, 0,
                             st>>>(a, first),
         note_launch());
    });
    if (L.ent_count > 0) {
        const int tpb = 256;
        (k_entry_scatter<R><<<dim3((unsigned)((L.ent_count + tpb - 1) / tpb), a.nf), tpb, 0, st>>>(a, L.ent_first,
                                                                                                  L.ent_count),
         note_launch());
    }
    if (L.max_piv <= 16)
        launch_mid<R, 16>(a, L, st);
    else
        launch_mid<R, NB>(a, L, st);
}

template bool mid_factor_level<double>(const LevelInfo &);
template bool mid_factor_level<float>(const LevelInfo &);
template void launch_factor_mid<double>(const FactorArgs<double> &, const LevelInfo &, cudaStream_t);
template void launch_factor_mid<float>(const FactorArgs<float> &, const LevelInfo &, cudaStream_t);

}  // namespace gm
