// Device-side argument blocks and launch wrappers shared by the engine.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/germaine_gpu.h"

namespace gm {

template <class R> struct cplx_any_t;
template <> struct cplx_any_t<double> { using type = double2; };
template <> struct cplx_any_t<float> { using type = float2; };
template <class R> using cplx_any = typename cplx_any_t<R>::type;

// Counts kernel launches of this library (reported in gm_stats).
void note_launch();
void note_launches(long long n);   // n kernels launched at once (a CUDA graph replay)
long long launch_count();

// ---------------- K1 assembly ----------------
struct AsmFreq {
    float2 om2;     // Omega^2 of the assembly
    float2 om;      // TE Omega
    float2 om2mu0;  // TE Omega^2 * mu0
    int model;      // material model of this matrix (index into [nmod][n])
    int pad;
};

struct AsmArgs {
    int nx, ny, n, nf, physics;
    float w[6];               // a, b, c, d, e, idh2
    const float *pml;         // [nf][pml_stride]
    int pml_stride;           // 4*(nx+2) + 4*(ny+2)
    const float *stiff;       // [nf][n]  b (AC) or mu (SH) of each matrix's model
    float2 *mass;             // [nf][n]
    double2 *A;               // [nf][9][n]
};

void launch_assemble(const AsmArgs &a, const float *m0, const float *m1, const AsmFreq *fq, float *stiff,
                     cudaStream_t st);

// ---------------- symbolic structure on the device ----------------
struct DevSym {
    int n, nnodes;
    const int *npiv, *nfront, *child0, *child1, *vars, *inv, *lvl_nodes;
    const int64_t *front_off, *var_off, *inv_off, *rhs_off;
    int64_t front_total, rhs_total;
};

// ---------------- K2-K4 numeric factorisation ----------------
struct LevelInfo {
    int first;      // offset into lvl_nodes
    int count;      // nodes in the level
    int max_front, max_piv, max_ring;
    int64_t ent_first, ent_count;  // level's entry range in ent_dst/ent_src
    int64_t mid_words;  // largest (f + 1) s + (s | 1)(f - s) of the level's fronts: k_factor_mid's tile
    int index;          // the level's height
};

// Launches that put a level's fronts on grid.y are split into pieces of at
// most kMaxGridY fronts (the hardware limit of gridDim.y); each piece passes
// its own first level position.
constexpr int kMaxGridY = 65535;
template <class F>
inline void for_level_pieces(const LevelInfo &L, F fn) {
    for (int c0 = 0; c0 < L.count; c0 += kMaxGridY) fn(L.first + c0, L.count - c0 < kMaxGridY ? L.count - c0 : kMaxGridY);
}

template <class R>
struct FactorArgs {
    DevSym s;
    void *front;              // cplx<R> [nf][front_total]
    const double2 *A;         // [nf][9][n] assembled stencil values
    const int64_t *ent_dst;   // per entry: front_off + position
    const int *ent_src;       // per entry: q*n + k into A (operator orientation applied)
    int nf;
    // static pivoting: |pivot| below pivscale * max|A| is replaced; max|A|
    // is a device scalar (bits of a non-negative double) written by
    // launch_amax, so the threshold never round-trips through the host
    const unsigned long long *amax;
    double pivscale;
    unsigned long long *npert;  // perturbed-pivot counter
    // threshold partial pivoting inside the 32-pivot blocks of the tiled
    // levels (fronts with more than NB pivots): pivtau2 = tolerance^2 (0 =
    // off); pivsrc[matrix * n + vars[k]] = the row of pivot k's block (0 ..
    // 31, equation order) that pivot position k took; nswap counts exchanges
    double pivtau2;
    unsigned char *pivsrc;
    unsigned long long *nswap;
    const int64_t *ent_lvl_off; // entries of level position t (index into lvl_nodes):
                                // ent_dst/ent_src[ent_lvl_off[t] .. ent_lvl_off[t + 1])
};

// max |A| over cnt complex entries into *out (bits of a double; *out must
// be zeroed first)
void launch_amax(const double2 *A, size_t cnt, unsigned long long *out, cudaStream_t st);
// dst[i] = (re[i], im[i])
void launch_pack_split(double2 *dst, const double *re, const double *im, size_t cnt, cudaStream_t st);

template <class R>
void launch_factor_level(const FactorArgs<R> &a, const LevelInfo &L, cudaStream_t st);
// Small fronts: the whole front of every node of the level assembled and
// factorised in shared memory by one CTA (replaces launch_factor_level and
// the level's contribution-block GEMM) when small_factor_level(L).
template <class R>
bool small_factor_level(const LevelInfo &L);
template <class R>
void launch_factor_small(const FactorArgs<R> &a, const LevelInfo &L, cudaStream_t st);
// Levels of fronts with at most NB pivots that do not fit the small kernel:
// gather, operator entries, then one CTA per front factorises the pivot
// panel in shared memory and applies the Schur update to the contribution
// block (replaces the K3 / K4 steps and the level's contribution GEMM).
template <class R>
bool mid_factor_level(const LevelInfo &L);
// the level's factorisation exchanges rows (FactorArgs::pivsrc) when
// pivoting is on: every level but the small-front kernel's
template <class R>
bool level_pivots(const LevelInfo &L);
template <class R>
void launch_factor_mid(const FactorArgs<R> &a, const LevelInfo &L, cudaStream_t st);


// one dense product C -= A * B (column-major, complex<R>)
template <class R>
struct GemmProb {
    const cplx_any<R> *A;
    const cplx_any<R> *B;
    cplx_any<R> *C;
    int lda, ldb, ldc, m, n, k;
};
// CUDA-core batched GEMM over 64 x 64 tiles: tiles[t] = (problem, tile row, tile col)
template <class R>
void launch_gemm_sub_cc(const GemmProb<R> *d_probs, const int4 *d_tiles, int ntiles, cudaStream_t st);
constexpr int kGemmTileCC = 64;

// ---------------- K5 multi-RHS substitution ----------------
template <class R>
struct SolveArgs {
    DevSym s;
    const void *front;        // cplx<R> factors [nf][front_total]
    void *x;                  // cplx<R> [nf][n][ldr], rhs in, solution out
    void *w;                  // cplx<R> [nf][rhs_total][ldr] update vectors (ring rows)
    int nf, nrhs, ldr;
    int rch;                  // right-hand sides per CTA (<= 32)
    int trans;                // 0: M x = b, 1: M^T x = b
    // forward-pass pruning (NULL: every front carries data): mask[v * mask_nch + g]
    // is 0 when right-hand sides 32 g .. 32 g + 31 are zero on every pivot row of
    // node v's subtree, so that node's y and update vector are zero
    const unsigned char *mask;
    int mask_nch;
    // matrices of this launch: fmap[0 .. nfz) (NULL: all nf, in order);
    // xmap[j]: slot of x / w for launch position j (NULL: the matrix index)
    const int *fmap;
    int nfz;
    const int *xmap;
    // live (front position in its level, slice) pairs of a pruned forward
    // pass (device), level h at work[work_off[h] .. work_off[h + 1]) (host
    // offsets), for slices of work_w[h] right-hand sides (host); NULL: no list
    const int2 *work;
    const int *work_off;
    const int *work_w;
    // host: per level {forward rt, forward B, backward rt, backward B} chosen
    // by the autotuner (gm_autotune; 0 entries keep the default rule), or NULL
    const int *lvl_cfg;
    // implicit spike right-hand sides (with a pruning mask only; NULL: x
    // holds b on entry): column r is spike_amp[matrix] on row spike_k[r] and
    // zero elsewhere.  x is not cleared beforehand: the forward pass writes
    // b + the children's updates at the pivot rows of every live front, and
    // the backward pass takes y = 0 at the pivot rows of pruned fronts.
    const int *spike_k;
    const double2 *spike_amp;
    // row exchanges of the factorisation's threshold pivoting (FactorArgs::
    // pivsrc; NULL: none): within each 32-pivot block of the fronts solved
    // by the ring / pivot kernels, the forward pass of M x = b gathers the
    // block's right-hand-side rows through it, the backward pass of
    // M^T x = b scatters the block's solution rows through it
    const unsigned char *pivsrc;
};

// right-hand sides per substitution slice for nrhs right-hand sides
int solve_slice_width(int nrhs, bool fp64);
// the built-in tile height of a level's substitution kernels (32 or 64)
int solve_level_rt(const LevelInfo &L);

template <class R>
void launch_solve_forward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st);
template <class R>
void launch_solve_backward_level(const SolveArgs<R> &a, const LevelInfo &L, cudaStream_t st);

// ---------------- K6 FP64 residual / refinement ----------------
struct ResidArgs {
    int nx, ny, n, nf, nrhs, ldr;
    const double2 *A;   // [nf][9][n]
    const double2 *x;   // [nf][n][ldr]
    const double2 *b;   // [nf][n][ldr]
    double2 *r;         // [nf][n][ldr] out: b - M x
    int op_mode;        // GM_OP_REF: M = A^T, GM_OP_EXACT: M = A
    int trans;          // 0: M, 1: M^T
    // spike right-hand sides given implicitly (b == NULL): b[f][k][r] =
    // spike_amp[f] if k == spike_k[r], else 0
    const int *spike_k;
    const double2 *spike_amp;
    // matrices of this launch: fmap[0 .. nfz) (NULL: all nf, in order);
    // partial sums and norms are indexed by the position in fmap
    const int *fmap;
    int nfz;
    // slots of x and of the output for launch position j (NULL: the
    // matrix index itself): xmap[j], omap[j]
    const int *xmap;
    const int *omap;
};
// row blocks of the residual kernel for n unknowns (the partial-sum count)
int residual_blocks(int nx, int ny);
// r = b - M x and per-(freq, rhs) partial sums of |r|^2 and |b|^2 into
// part[nblk][nfz][nrhs][2]; returns nblk.
int launch_residual(const ResidArgs &a, double *part, int max_blocks, cudaStream_t st);
void launch_reduce_norms(const double *part, int nblk, int cnt, double *out, cudaStream_t st);
// as launch_residual, but writes (T)(b - M'x) into t [nf][n][ldr] instead of r
// (t = NULL: the norms only)
template <class R>
int launch_residual_t(const ResidArgs &a, void *t, double *part, int max_blocks, cudaStream_t st);
// out = M' x (FP64) for x of working precision cplx<R>, with the partial
// sums of |out|^2 (b ignored; the |b|^2 sums are 0)
template <class R>
int launch_matvec(const ResidArgs &a, const void *x, double2 *out, double *part, int max_blocks, cudaStream_t st);

// y(T) <- x(double) and x(double) += d(T) over [nf][n][ldr]
template <class R>
void launch_convert_down(const double2 *src, void *dst, size_t count, cudaStream_t st);
template <class R>
void launch_add_up(double2 *x, const void *d, size_t count, cudaStream_t st);
// x[f] += d[f] for the matrices f = fmap[0 .. nfz) (device list), per_f entries each
template <class R>
void launch_add_up_f(double2 *x, const void *d, size_t per_f, const int *fmap, int nfz, cudaStream_t st);

// ---------------- K6b GMRES-IR vector kernels ----------------
// Vectors [slot][n][nrhs]; j indexes the launch's list (zmap: slots, fmap:
// matrices of the batch); per-column coefficient arrays are
// [j][nrhs][kGmresStride] complex.
constexpr int kGmresMaxRestart = 8;
constexpr int kGmresStride = kGmresMaxRestart + 1;
// Z[zmap[j]] = (R)(V[zmap[j]] * s[j][r])
template <class R>
void launch_scale_down(const double2 *V, void *Z, const double *s, const int *zmap, int nj, int n, int nrhs,
                       cudaStream_t st);
// part[blk][j][r][0 .. nv] = partial sums of conj(V_i) W (i < nv) and |W|^2;
// V_i = V + i * vstride; returns the number of row blocks
int launch_dots(const double2 *V, size_t vstride, int nv, const double2 *W, const int *zmap, int nj, int n, int nrhs,
                double *part, cudaStream_t st);
// W -= sum_i coef[j][r][i] V_i; part[blk][j][r] = partial sums of |W|^2
int launch_gs_update(const double2 *V, size_t vstride, int nv, double2 *W, const double2 *coef, const int *zmap,
                     int nj, int n, int nrhs, double *part, cudaStream_t st);
// x[fmap[j]] += sum_{i < nz} y[j][r][i] Z_i[zmap[j]]
template <class R>
void launch_x_update(double2 *x, const void *Z, size_t zstride, int nz, const double2 *y, const int *fmap,
                     const int *zmap, int nj, int n, int nrhs, cudaStream_t st);
void preload_gmres_kernels();

// Load every substitution / refinement kernel now (lazy module loading
// would otherwise load each on its first launch, taking device memory).
void preload_solve_kernels();
void preload_refine_kernels();

// one ordered float dot product (lbfgs.cu: k_dot_seq): out = sum a[i] * b[i], i = 0..n-1 in order
struct DotJob {
    const float *a, *b;
    long n;
    float *out;
};

}  // namespace gm
