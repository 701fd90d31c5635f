// K6: FP64 residual r = b - M x of the 9-point operator for every
// right-hand side of every frequency, with per-(frequency, right-hand side)
// partial sums of |r|^2 and |b|^2, and the precision conversions of the
// mixed-precision refinement loop.  HBM-bound: per row 9 operator values
// (amortised over the right-hand sides) and x, b, r for each right-hand side.
#include <cstdlib>
#include "kernels.cuh"
#include "cplx.cuh"

namespace gm {

// Residual tile: a patch of PL grid lines x PW grid columns of one matrix x
// RLANES right-hand sides.  Warp w walks grid line y0 + w of the patch from
// left to right, one grid point per step, with the 3 x 3 stencil window of
// x in registers: each step loads only the window's new right-hand column
// (the points above, at and below the next grid point: three 512-byte
// loads per step, RSTEP steps' loads issued together), so every x value is
// loaded by three warps of the patch or its neighbours instead of nine
// times.  The vertical neighbours of a warp's line are the centre lines of
// the warps above and below it, so most of them come from L1.  The
// patch's operator values (9 per grid point, shared by every right-hand
// side; zero for neighbours outside the grid, so the stencil needs no
// edge branches) are staged in shared memory once.
constexpr int PW = 32;      // grid columns per patch (steps per warp)
constexpr int PL = 8;       // grid lines per patch (warps per CTA)
constexpr int RLANES = 32;  // right-hand sides per CTA
constexpr int RSTEP = 3;    // window steps whose loads are in flight together
static_assert(PW == RLANES, "one patch point per thread when the patch is staged");

// patches of the residual kernel on an nx x ny grid (partial-sum blocks)
int residual_blocks(int nx, int ny) { return ((nx + PW - 1) / PW) * ((ny + PL - 1) / PL); }

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
// SEG = 1: lane = right-hand side r0 + lane, each warp walking its whole
// line segment of the patch.  SEG > 1 (the last few right-hand sides, when
// fewer than RLANES are left): lane = (segment, right-hand side), 32 / SEG
// right-hand sides from r0, each lane walking PW / SEG points of its line
// -- a warp instruction then serves SEG times the points where one lane per
// right-hand side would leave most of the warp idle.
template <class InC, class OutC, bool WRITE, bool PRODUCT, int SEG>
__global__ void __launch_bounds__(RLANES *PL, 2) k_residual(ResidArgs a, const InC *__restrict__ xin, OutC *out,
                                                          double *part, int r0) {
    constexpr int RL = RLANES / SEG, SW = PW / SEG;   // right-hand sides per warp, points per lane
    __shared__ double2 cf[9][PL][PW];   // operator values, zero for neighbours outside the grid
    __shared__ double red[2][PL][RLANES];
    const int fz = blockIdx.z;
    const int f = a.fmap ? a.fmap[fz] : fz;
    const int ncb = (a.nx + PW - 1) / PW;
    const int x0 = (int)(blockIdx.x % ncb) * PW, y0 = (int)(blockIdx.x / ncb) * PL;
    const int r = r0 + blockIdx.y * RL + threadIdx.x % RL;
    const int seg = threadIdx.x / RL;
    const bool use_row = (a.op_mode == GM_OP_EXACT) != (a.trans != 0);
    const double2 *A9 = a.A + (size_t)f * 9 * a.n;
    {   // one grid point of the patch per thread: its operator values
        const int ly = threadIdx.y, lx = threadIdx.x;
        const int x = x0 + lx, y = y0 + ly;
        unsigned m = 0;   // bit q: neighbour q lies inside the grid
        if (x < a.nx && y < a.ny) {
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const int xx = x + q % 3 - 1, yy = y + q / 3 - 1;
                if (xx >= 0 && xx < a.nx && yy >= 0 && yy < a.ny) m |= 1u << q;
            }
        }
        const int k = y * a.nx + x;
#pragma unroll
        for (int q = 0; q < 9; ++q)
            cf[q][ly][lx] = (m >> q) & 1 ? op_coef(A9, a.n, a.nx, use_row, q, k) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double rr = 0.0, bb = 0.0;
    const int w = threadIdx.y, y = y0 + w;
    const int xs = seg * SW, xe = min(xs + SW, a.nx - x0);   // this lane's columns of the patch
    if (r < a.nrhs && y < a.ny && xs < xe) {
        const size_t per = (size_t)a.n * a.ldr;
        const size_t base = (size_t)f * per + r;
        const size_t ldr = a.ldr;
        const InC *X = xin + (size_t)(a.xmap ? a.xmap[fz] : f) * per + r;
        OutC *O = out ? out + (size_t)(a.omap ? a.omap[fz] : f) * per + r : nullptr;
        const bool spikes = !PRODUCT && a.spike_k;
        const int ks = spikes ? a.spike_k[r] : -1;
        const double2 amp = spikes ? a.spike_amp[f] : make_double2(0.0, 0.0);
        const int n = a.n, nx = a.nx;
        // x at flat index i, zero outside the array (such values are masked)
        auto ld = [&](int i) { return (i >= 0 && i < n) ? cto_d(X[(size_t)i * ldr]) : make_double2(0.0, 0.0); };
        const int kb = y * nx + x0 + xs;   // flat index of the lane's first point
        // window: wl[d] / wc[d] = x left of / at the current point on the
        // line above (d = 0), the same line (1) and the line below (2)
        double2 wl[3], wc[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            wl[d] = ld(kb - 1 + (d - 1) * nx);
            wc[d] = ld(kb + (d - 1) * nx);
        }
        const int ne = xe - xs;   // points of this lane
        for (int c0 = 0; c0 < ne; c0 += RSTEP) {
            double2 wr[RSTEP][3];   // the right-hand columns of the next RSTEP points
#pragma unroll
            for (int u = 0; u < RSTEP; ++u)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    wr[u][d] = c0 + u < ne ? ld(kb + c0 + u + 1 + (d - 1) * nx) : make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < RSTEP; ++u) {
                const int lx = xs + c0 + u;   // column in the patch
                if (c0 + u >= ne) break;
                const int k = kb + c0 + u;
                double2 bv = make_double2(0.0, 0.0);
                if (!PRODUCT) bv = spikes ? (k == ks ? amp : bv) : a.b[base + (size_t)k * ldr];
                double2 acc = bv;
                // no branches on the grid edges: a neighbour outside the grid
                // has a zero operator value, and acc - 0 x is acc exactly
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    cfms(acc, cf[3 * d][w][lx], wl[d]);
                    cfms(acc, cf[3 * d + 1][w][lx], wc[d]);
                    cfms(acc, cf[3 * d + 2][w][lx], wr[u][d]);
                }
                if (PRODUCT) acc = make_double2(-acc.x, -acc.y);
                if (WRITE) O[(size_t)k * ldr] = cconv<OutC>(acc);
                rr += acc.x * acc.x + acc.y * acc.y;
                bb += bv.x * bv.x + bv.y * bv.y;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    wl[d] = wc[d];
                    wc[d] = wr[u][d];
                }
            }
        }
    }
    red[0][w][threadIdx.x] = rr;
    red[1][w][threadIdx.x] = bb;
    __syncthreads();
    if (threadIdx.y == 0 && threadIdx.x < RL && r < a.nrhs) {   // fixed order: deterministic
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int g = 0; g < PL; ++g)
#pragma unroll
            for (int q = 0; q < SEG; ++q) {
                s0 += red[0][g][q * RL + threadIdx.x];
                s1 += red[1][g][q * RL + threadIdx.x];
            }
        double *p = part + (((size_t)blockIdx.x * gridDim.z + fz) * a.nrhs + r) * 2;
        p[0] = s0;
        p[1] = s1;
    }
}

static int resid_nfz(const ResidArgs &a) { return a.fmap ? a.nfz : a.nf; }

// Full groups of RLANES right-hand sides, then the rest (at most 8) by the
// segmented form; the partial sums land in the same slots either way.
template <class InC, class OutC, bool WRITE, bool PRODUCT>
static int launch_k6(const ResidArgs &a, const void *x, void *out, double *part, int max_blocks, cudaStream_t st) {
    const int nblk = residual_blocks(a.nx, a.ny);
    const int nfz = resid_nfz(a);
    if (nblk > max_blocks) return -1;
    if (nfz <= 0) return nblk;
    static const bool no_tail = [] {   // GM_NO_TAIL_SLICE=1: one lane per right-hand side throughout
        const char *v = std::getenv("GM_NO_TAIL_SLICE");
        return v && std::atoi(v) != 0;
    }();
    const int rem = a.nrhs % RLANES;
    const int tail = no_tail || rem == 0 || rem > 8 ? 0 : rem;
    const int nfull = (a.nrhs - tail + RLANES - 1) / RLANES;
    const InC *xi = reinterpret_cast<const InC *>(x);
    OutC *o = reinterpret_cast<OutC *>(out);
    if (nfull > 0)
        (k_residual<InC, OutC, WRITE, PRODUCT, 1><<<dim3(nblk, nfull, nfz), dim3(RLANES, PL), 0, st>>>(a, xi, o, part, 0),
         note_launch());
    if (tail > 4)
        (k_residual<InC, OutC, WRITE, PRODUCT, 4><<<dim3(nblk, 1, nfz), dim3(RLANES, PL), 0, st>>>(
             a, xi, o, part, RLANES * nfull),
         note_launch());
    else if (tail > 0)
        (k_residual<InC, OutC, WRITE, PRODUCT, 8><<<dim3(nblk, 1, nfz), dim3(RLANES, PL), 0, st>>>(
             a, xi, o, part, RLANES * nfull),
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
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, double2, true, false, 1>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, double2, false, false, 1>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, float2, true, false, 1>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, float2, false, false, 1>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, double2, true, false, 4>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, double2, false, false, 4>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, float2, true, false, 4>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, float2, false, false, 4>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, double2, true, false, 8>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, double2, false, false, 8>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, float2, true, false, 8>);
    cudaFuncGetAttributes(&fa, (const void *)k_residual<double2, float2, false, false, 8>);
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
