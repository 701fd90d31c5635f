// Quasi-Newton l-BFGS update of the reference on the device, with the
// history resident in HBM: LBFGS (src/LBFGS.c:12-250, one parameter class)
// and LBFGS_TE (src/TE/LBFGS_TE.c, two classes sigma / epsilon, optionally
// scaled by the diagonal Hessians), rot_LBFGS_vec, zero_LBFGS,
// check_descent / check_descent_multi_para_TE and calc_mat_change_wolfe /
// calc_mat_change_wolfe_multi_para.
//
// Results are bit-identical to the reference's float arithmetic.  Its dot
// products (dotp, src/dotp.c:10-35; dotp_matrix) add rounded float products
// one after the other; that order is kept: one warp per dot product forms
// 32 products at a time in parallel and every lane runs the same ordered
// chain of float additions over them (shuffle broadcast), so a dot product
// costs one dependent add per element.  Independent dot products run as
// separate warps of one launch.  Everything else is elementwise in HBM.
//
// Vectors are kept in the reference's order: class outer, then x outer, y
// inner (h = c * NX * NY + i * NY + j); callers pass [nclass][NY][NX]
// row-major grids.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.hpp"
#include "germaine_gpu.h"
#include "host_setup.h"
#include "kernels.cuh"

struct gm_lbfgs {
    int device = 0, nx = 0, ny = 0, npml = 0, free_surf = 0, nclass = 1, m = 1;
    size_t n = 0, nvec = 0;
    cudaStream_t st = nullptr;
    float *y = nullptr, *s = nullptr;             // [m][nvec]
    float *old_grad = nullptr, *old_model = nullptr;   // [nvec] the "*.old" file contents
    float *q = nullptr, *r = nullptr, *t0 = nullptr, *t1 = nullptr;   // [nvec] work vectors
    float *grid = nullptr;                        // [nvec] staging of caller grids
    float *sums = nullptr;                        // dot products: [0] nom [1] den, [2..] per slot
    float *coef = nullptr;                        // frame taper coefficient [n]
    unsigned char *passes = nullptr;              // frame taper multiplicity [n]
    unsigned *maxbits = nullptr;                  // |hess| maxima per class
    gm::DotJob *jobs = nullptr;                   // device job list
    bool have_old = false;
};

namespace gm {

// ---- ordered float dot product, one warp per job ----
__global__ void __launch_bounds__(32) k_dot_seq(const DotJob *__restrict__ jobs) {
    const DotJob jb = jobs[blockIdx.x];
    const int lane = threadIdx.x;
    const float *__restrict__ a = jb.a;
    const float *__restrict__ b = jb.b;
    const long n = jb.n;
    float acc = 0.0f;
    constexpr int U = 4;   // chunks of 32 loaded ahead
    float p[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const long i = (long)u * 32 + lane;
        p[u] = i < n ? __fmul_rn(__ldg(a + i), __ldg(b + i)) : 0.0f;
    }
    for (long base = 0; base < n; base += 32 * U) {
        float pn[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long i = base + 32 * U + (long)u * 32 + lane;
            pn[u] = i < n ? __fmul_rn(__ldg(a + i), __ldg(b + i)) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long c0 = base + (long)u * 32;
            if (c0 + 32 <= n) {
#pragma unroll
                for (int t = 0; t < 32; ++t) acc = __fadd_rn(acc, __shfl_sync(0xffffffffu, p[u], t));
            } else {
                const int cnt = c0 < n ? (int)(n - c0) : 0;
                for (int t = 0; t < 32; ++t) {
                    const float v = __shfl_sync(0xffffffffu, p[u], t);
                    if (t < cnt) acc = __fadd_rn(acc, v);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) p[u] = pn[u];
    }
    if (lane == 0) *jb.out = acc;
}

// rho of slot k as the reference forms it (src/LBFGS.c:86-91): 1.0 / sum in
// double, stored as float; 0 for a zero sum
__device__ __forceinline__ float lbfgs_rho(float sum) {
    return fabsf(sum) > 0.0f ? __double2float_rn(__ddiv_rn(1.0, (double)sum)) : 0.0f;
}

// grid [nclass][ny][nx] <-> vector h = c * n + i * ny + j
__device__ __forceinline__ size_t grid_index(size_t h, size_t n, int nx, int ny) {
    const size_t c = h / n, rem = h % n;
    const int i = (int)(rem / ny), j = (int)(rem % ny);
    return c * n + (size_t)j * nx + i;
}

__global__ void k_to_vec(const float *__restrict__ grid, float *__restrict__ v, size_t nvec, size_t n, int nx, int ny) {
    const size_t h = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h < nvec) v[h] = grid[grid_index(h, n, nx, ny)];
}

__global__ void k_to_grid(const float *__restrict__ v, float *__restrict__ grid, size_t nvec, size_t n, int nx, int ny) {
    const size_t h = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h < nvec) grid[grid_index(h, n, nx, ny)] = v[h];
}

// y = grad - old_grad, s = model - old_model (src/LBFGS.c:54-60)
__global__ void k_lbfgs_ys(const float *__restrict__ grad, const float *__restrict__ model,
                           const float *__restrict__ og, const float *__restrict__ om, float *__restrict__ y,
                           float *__restrict__ s, size_t nvec, size_t n, int nx, int ny) {
    const size_t h = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nvec) return;
    const size_t g = grid_index(h, n, nx, ny);
    y[h] = __fsub_rn(grad[g], og[h]);
    s[h] = __fsub_rn(model[g], om[h]);
}

// q -= alpha_k y_k with alpha_k = rho_k * (s_k . q) (src/LBFGS.c:109-123)
__global__ void k_lbfgs_q(float *__restrict__ q, const float *__restrict__ yk, const float *__restrict__ sums,
                          int k, int m, size_t nvec) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nvec) return;
    const float alpha = __fmul_rn(lbfgs_rho(sums[2 + k]), sums[2 + m + k]);
    q[i] = __fsub_rn(q[i], __fmul_rn(alpha, yk[i]));
}

// r = gamma q (src/LBFGS.c:124-126), or q / (hess + EPS_HESS * MAX_HESS)
// per class (src/TE/LBFGS_TE.c, HESSIAN != 0)
__global__ void k_lbfgs_r0(const float *__restrict__ q, float *__restrict__ r, const float *__restrict__ sums,
                           const float *__restrict__ hess, float eps_hess, const unsigned *__restrict__ maxbits,
                           size_t nvec, size_t n, int nx, int ny) {
    const size_t h = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nvec) return;
    if (!hess) {
        r[h] = __fmul_rn(__fdiv_rn(sums[0], sums[1]), q[h]);
    } else {
        const float em = __fmul_rn(eps_hess, __uint_as_float(maxbits[h / n]));
        r[h] = __fdiv_rn(q[h], __fadd_rn(hess[grid_index(h, n, nx, ny)], em));
    }
}

// r += s_k (alpha_k - beta_k), beta_k = rho_k * (y_k . r) (src/LBFGS.c:129-144)
__global__ void k_lbfgs_r(float *__restrict__ r, const float *__restrict__ sk, const float *__restrict__ sums, int k,
                          int m, size_t nvec) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nvec) return;
    const float rho = lbfgs_rho(sums[2 + k]);
    const float alpha = __fmul_rn(rho, sums[2 + m + k]);
    const float beta = __fmul_rn(rho, sums[2 + 2 * m + k]);
    r[i] = __fadd_rn(r[i], __fmul_rn(sk[i], __fsub_rn(alpha, beta)));
}

// cp_grad_frame on float grids (src/cp_grad_frame.c:162-208): each frame
// strip that covers a point multiplies it by the point's coefficient, in float
__global__ void k_taper_float(float *__restrict__ g, const float *__restrict__ coef,
                              const unsigned char *__restrict__ passes, size_t n, int nclass) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * nclass) return;
    const size_t k = t % n;
    float v = g[t];
    const float c = coef[k];
    for (int p = passes[k]; p > 0; --p) v = __fmul_rn(v, c);
    g[t] = v;
}

__global__ void __launch_bounds__(256) k_abs_max(const float *__restrict__ x, size_t n, unsigned *maxbits) {
    float m = 0.0f;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[k]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxbits, __float_as_uint(m));
}

// calc_mat_change_wolfe (mode 0, src/calc_mat_change_wolfe.c:27-47): a value
// outside [low, up] or below zero falls back to the old one;
// calc_mat_change_wolfe_multi_para (mode 1): clamped to [low, up]
__global__ void k_mat_change(const float *__restrict__ hgrad, const float *__restrict__ old, float *__restrict__ out,
                             size_t n, float eps_scale, float low, float up, int mode) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float o = old[k];
    float v = __fadd_rn(o, __fmul_rn(eps_scale, hgrad[k]));
    if (mode == 0) {
        if (v < low) v = o;
        if (v > up) v = o;
        if (v < 0.0f) v = o;
    } else {
        if (v < low) v = low;
        if (v > up) v = up;
    }
    out[k] = v;
}

}  // namespace gm

namespace {

constexpr int TPB = 256;

unsigned blocks(size_t n) { return (unsigned)((n + TPB - 1) / TPB); }

int cuda_fail(cudaError_t e, const char *what) {
    return gm::fail(e == cudaErrorMemoryAllocation ? GM_ERROR_OUT_OF_MEMORY : GM_ERROR_CUDA, "%s: %s", what,
                    cudaGetErrorString(e));
}

#define LB_CUDA(call, what)                          \
    do {                                             \
        cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// copy a caller buffer (host or device) of count floats into dst on the stream
int stage(gm_lbfgs *h, float *dst, const float *src, size_t count, const char *what) {
    LB_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyDefault, h->st), what);
    return GM_OK;
}

int run_dots(gm_lbfgs *h, const std::vector<gm::DotJob> &jobs) {
    LB_CUDA(cudaMemcpyAsync(h->jobs, jobs.data(), jobs.size() * sizeof(gm::DotJob), cudaMemcpyHostToDevice, h->st),
            "l-BFGS dot jobs");
    gm::k_dot_seq<<<(unsigned)jobs.size(), 32, 0, h->st>>>(h->jobs);
    gm::note_launch();
    LB_CUDA(cudaGetLastError(), "l-BFGS dot products");
    // the job list is reused by the next launch: keep the host copy alive until it is consumed
    LB_CUDA(cudaStreamSynchronize(h->st), "l-BFGS dot products");
    return GM_OK;
}

}  // namespace

extern "C" int gm_lbfgs_create(int device, int nx, int ny, int npml, int free_surf, int nclass, int m,
                               gm_lbfgs **out) {
    if (!out) return gm::fail(GM_ERROR_INVALID, "gm_lbfgs_create: null output");
    *out = nullptr;
    if (nx <= 0 || ny <= 0 || npml < 0 || (nclass != 1 && nclass != 2) || m <= 0)
        return gm::fail(GM_ERROR_INVALID, "gm_lbfgs_create: bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_lbfgs_create: bad device %d", device);
    auto *h = new (std::nothrow) gm_lbfgs();
    if (!h) return gm::fail(GM_ERROR_OUT_OF_MEMORY, "gm_lbfgs_create: host allocation failed");
    h->device = device; h->nx = nx; h->ny = ny; h->npml = npml; h->free_surf = free_surf;
    h->nclass = nclass; h->m = m;
    h->n = (size_t)nx * ny;
    h->nvec = h->n * nclass;
    const size_t vb = h->nvec * sizeof(float);
    cudaError_t e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&h->y, vb * m);
    if (e == cudaSuccess) e = cudaMalloc(&h->s, vb * m);
    if (e == cudaSuccess) e = cudaMalloc(&h->old_grad, vb);
    if (e == cudaSuccess) e = cudaMalloc(&h->old_model, vb);
    if (e == cudaSuccess) e = cudaMalloc(&h->q, vb);
    if (e == cudaSuccess) e = cudaMalloc(&h->r, vb);
    if (e == cudaSuccess) e = cudaMalloc(&h->t0, vb);
    if (e == cudaSuccess) e = cudaMalloc(&h->t1, vb);
    if (e == cudaSuccess) e = cudaMalloc(&h->grid, vb);
    if (e == cudaSuccess) e = cudaMalloc(&h->sums, (2 + 3 * (size_t)m + 8) * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&h->coef, h->n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&h->passes, h->n);
    if (e == cudaSuccess) e = cudaMalloc(&h->maxbits, 2 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&h->jobs, (2 + (size_t)m) * sizeof(gm::DotJob));
    if (e == cudaSuccess) e = cudaMemset(h->y, 0, vb * m);
    if (e == cudaSuccess) e = cudaMemset(h->s, 0, vb * m);
    if (e == cudaSuccess) {
        std::vector<float> coef(h->n);
        std::vector<unsigned char> passes(h->n);
        gmh_grad_frame(nx, ny, npml, free_surf, coef.data(), passes.data());
        e = cudaMemcpy(h->coef, coef.data(), h->n * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->passes, passes.data(), h->n, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        const int rc = cuda_fail(e, "gm_lbfgs_create");
        gm_lbfgs_destroy(h);
        return rc;
    }
    *out = h;
    return GM_OK;
}

extern "C" int gm_lbfgs_destroy(gm_lbfgs *h) {
    if (!h) return GM_OK;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    for (void *p : {(void *)h->y, (void *)h->s, (void *)h->old_grad, (void *)h->old_model, (void *)h->q, (void *)h->r,
                    (void *)h->t0, (void *)h->t1, (void *)h->grid, (void *)h->sums, (void *)h->coef,
                    (void *)h->passes, (void *)h->maxbits, (void *)h->jobs})
        if (p) cudaFree(p);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
    return GM_OK;
}

extern "C" int gm_lbfgs_step(gm_lbfgs *h, int first, int pointer, const float *grad, const float *gradm,
                             const float *model, const float *hess, float eps_hess, float *hgrad) {
    if (!h || !grad || !gradm || !model || !hgrad) return gm::fail(GM_ERROR_INVALID, "gm_lbfgs_step: bad argument");
    if (!first && (pointer < 1 || pointer > h->m))
        return gm::fail(GM_ERROR_INVALID, "gm_lbfgs_step: pointer %d outside 1..%d", pointer, h->m);
    if (!first && !h->have_old)
        return gm::fail(GM_ERROR_STATE, "gm_lbfgs_step: no previous gradient and model (first step, or gm_lbfgs_set_old)");
    LB_CUDA(cudaSetDevice(h->device), "gm_lbfgs_step");
    const size_t nvec = h->nvec, n = h->n;
    const int m = h->m, nx = h->nx, ny = h->ny;
    int rc;
    float *gstage = h->t0, *mstage = h->t1;   // caller grids staged as given (row-major)
    if ((rc = stage(h, gstage, grad, nvec, "gm_lbfgs_step: gradient"))) return rc;
    if ((rc = stage(h, mstage, model, nvec, "gm_lbfgs_step: model"))) return rc;
    if ((rc = stage(h, h->grid, gradm, nvec, "gm_lbfgs_step: preconditioned gradient"))) return rc;
    float *out = h->grid;   // row-major result, tapered in place
    if (!first) {
        float *yp = h->y + (size_t)(pointer - 1) * nvec, *sp = h->s + (size_t)(pointer - 1) * nvec;
        gm::k_lbfgs_ys<<<blocks(nvec), TPB, 0, h->st>>>(gstage, mstage, h->old_grad, h->old_model, yp, sp, nvec, n,
                                                          nx, ny);
        gm::note_launch();
        // gamma and every slot's rho: independent dot products in one launch
        std::vector<gm::DotJob> jobs;
        jobs.push_back({yp, sp, (long)nvec, h->sums + 0});
        jobs.push_back({yp, yp, (long)nvec, h->sums + 1});
        for (int k = 0; k < m; ++k)
            jobs.push_back({h->y + (size_t)k * nvec, h->s + (size_t)k * nvec, (long)nvec, h->sums + 2 + k});
        if ((rc = run_dots(h, jobs))) return rc;
        gm::k_to_vec<<<blocks(nvec), TPB, 0, h->st>>>(h->grid, h->q, nvec, n, nx, ny);
        gm::note_launch();
        for (int k = m - 1; k >= 0; --k) {
            if ((rc = run_dots(h, {{h->s + (size_t)k * nvec, h->q, (long)nvec, h->sums + 2 + m + k}}))) return rc;
            gm::k_lbfgs_q<<<blocks(nvec), TPB, 0, h->st>>>(h->q, h->y + (size_t)k * nvec, h->sums, k, m, nvec);
            gm::note_launch();
        }
        const float *dhess = nullptr;
        if (hess) {
            if ((rc = stage(h, h->t0, hess, nvec, "gm_lbfgs_step: Hessian"))) return rc;
            LB_CUDA(cudaMemsetAsync(h->maxbits, 0, 2 * sizeof(unsigned), h->st), "gm_lbfgs_step");
            for (int c = 0; c < h->nclass; ++c) {
                gm::k_abs_max<<<(unsigned)std::min<size_t>(blocks(n), 148 * 8), TPB, 0, h->st>>>(h->t0 + c * n, n,
                                                                                                  h->maxbits + c);
                gm::note_launch();
            }
            dhess = h->t0;
        }
        gm::k_lbfgs_r0<<<blocks(nvec), TPB, 0, h->st>>>(h->q, h->r, h->sums, dhess, eps_hess, h->maxbits, nvec, n,
                                                          nx, ny);
        gm::note_launch();
        for (int k = 0; k < m; ++k) {
            if ((rc = run_dots(h, {{h->y + (size_t)k * nvec, h->r, (long)nvec, h->sums + 2 + 2 * m + k}}))) return rc;
            gm::k_lbfgs_r<<<blocks(nvec), TPB, 0, h->st>>>(h->r, h->s + (size_t)k * nvec, h->sums, k, m, nvec);
            gm::note_launch();
        }
        gm::k_to_grid<<<blocks(nvec), TPB, 0, h->st>>>(h->r, out, nvec, n, nx, ny);
        gm::note_launch();
        // the model staging is reread below: restage the gradient (t0 held the Hessian)
        if (hess && (rc = stage(h, gstage, grad, nvec, "gm_lbfgs_step: gradient"))) return rc;
    }
    gm::k_taper_float<<<blocks(nvec), TPB, 0, h->st>>>(out, h->coef, h->passes, n, h->nclass);
    gm::note_launch();
    // this call's gradient and model become the "*.old" state
    gm::k_to_vec<<<blocks(nvec), TPB, 0, h->st>>>(gstage, h->old_grad, nvec, n, nx, ny);
    gm::note_launch();
    gm::k_to_vec<<<blocks(nvec), TPB, 0, h->st>>>(mstage, h->old_model, nvec, n, nx, ny);
    gm::note_launch();
    LB_CUDA(cudaMemcpyAsync(hgrad, out, nvec * sizeof(float), cudaMemcpyDefault, h->st), "gm_lbfgs_step: result");
    LB_CUDA(cudaStreamSynchronize(h->st), "gm_lbfgs_step");
    h->have_old = true;
    return GM_OK;
}

extern "C" int gm_lbfgs_rotate(gm_lbfgs *h) {
    if (!h) return gm::fail(GM_ERROR_INVALID, "gm_lbfgs_rotate: null handle");
    LB_CUDA(cudaSetDevice(h->device), "gm_lbfgs_rotate");
    const size_t bytes = (size_t)(h->m - 1) * h->nvec * sizeof(float);
    if (bytes) {   // slots 2..m move down one, slot by slot in order (slot m keeps its contents)
        for (int k = 1; k < h->m; ++k) {
            LB_CUDA(cudaMemcpyAsync(h->y + (size_t)(k - 1) * h->nvec, h->y + (size_t)k * h->nvec,
                                    h->nvec * sizeof(float), cudaMemcpyDeviceToDevice, h->st),
                    "gm_lbfgs_rotate");
            LB_CUDA(cudaMemcpyAsync(h->s + (size_t)(k - 1) * h->nvec, h->s + (size_t)k * h->nvec,
                                    h->nvec * sizeof(float), cudaMemcpyDeviceToDevice, h->st),
                    "gm_lbfgs_rotate");
        }
    }
    LB_CUDA(cudaStreamSynchronize(h->st), "gm_lbfgs_rotate");
    return GM_OK;
}

extern "C" int gm_lbfgs_zero(gm_lbfgs *h) {
    if (!h) return gm::fail(GM_ERROR_INVALID, "gm_lbfgs_zero: null handle");
    LB_CUDA(cudaSetDevice(h->device), "gm_lbfgs_zero");
    LB_CUDA(cudaMemsetAsync(h->y, 0, (size_t)h->m * h->nvec * sizeof(float), h->st), "gm_lbfgs_zero");
    LB_CUDA(cudaMemsetAsync(h->s, 0, (size_t)h->m * h->nvec * sizeof(float), h->st), "gm_lbfgs_zero");
    LB_CUDA(cudaStreamSynchronize(h->st), "gm_lbfgs_zero");
    return GM_OK;
}

extern "C" int gm_lbfgs_check_descent(gm_lbfgs *h, const float *hgrad, const float *grad, float *p_out) {
    if (!h || !hgrad || !grad) return gm::fail(GM_ERROR_INVALID, "gm_lbfgs_check_descent: bad argument");
    LB_CUDA(cudaSetDevice(h->device), "gm_lbfgs_check_descent");
    const size_t nvec = h->nvec, n = h->n;
    int rc;
    // dotp_matrix order (x outer, y inner) per class: stage both grids as vectors
    if ((rc = stage(h, h->grid, hgrad, nvec, "gm_lbfgs_check_descent: direction"))) return rc;
    gm::k_to_vec<<<blocks(nvec), TPB, 0, h->st>>>(h->grid, h->q, nvec, n, h->nx, h->ny);
    gm::note_launch();
    if ((rc = stage(h, h->grid, grad, nvec, "gm_lbfgs_check_descent: gradient"))) return rc;
    gm::k_to_vec<<<blocks(nvec), TPB, 0, h->st>>>(h->grid, h->r, nvec, n, h->nx, h->ny);
    gm::note_launch();
    float *sums = h->sums + 2 + 3 * (size_t)h->m;   // 4 spare slots
    std::vector<gm::DotJob> jobs;
    for (int c = 0; c < h->nclass; ++c) {
        jobs.push_back({h->q + c * n, h->r + c * n, (long)n, sums + c});
        jobs.push_back({h->r + c * n, h->r + c * n, (long)n, sums + 2 + c});
    }
    if ((rc = run_dots(h, jobs))) return rc;
    float v[4] = {0, 0, 0, 0};
    LB_CUDA(cudaMemcpy(v, sums, 4 * sizeof(float), cudaMemcpyDeviceToHost), "gm_lbfgs_check_descent");
    // check_descent (src/check_descent.c:17-19); for two classes the class
    // sums are added in float (src/TE/check_descent_multi_para_TE.c:21-26)
    float nom = v[0], den = v[2];
    if (h->nclass == 2) {
        nom = nom + v[1];
        den = den + v[3];
    }
    const float p = -nom / den;
    if (p_out) *p_out = p;
    if (p < 0.0f) return gm_lbfgs_zero(h);   // loss of descent: reset the history
    return GM_OK;
}

extern "C" int gm_lbfgs_get_old(gm_lbfgs *h, float *grad_old, float *model_old) {
    if (!h) return gm::fail(GM_ERROR_INVALID, "gm_lbfgs_get_old: null handle");
    if (!h->have_old) return gm::fail(GM_ERROR_STATE, "gm_lbfgs_get_old: no step taken yet");
    LB_CUDA(cudaSetDevice(h->device), "gm_lbfgs_get_old");
    const size_t nvec = h->nvec;
    for (int w = 0; w < 2; ++w) {
        float *dst = w ? model_old : grad_old;
        if (!dst) continue;
        gm::k_to_grid<<<blocks(nvec), TPB, 0, h->st>>>(w ? h->old_model : h->old_grad, h->grid, nvec, h->n, h->nx,
                                                         h->ny);
        gm::note_launch();
        LB_CUDA(cudaMemcpyAsync(dst, h->grid, nvec * sizeof(float), cudaMemcpyDefault, h->st), "gm_lbfgs_get_old");
        LB_CUDA(cudaStreamSynchronize(h->st), "gm_lbfgs_get_old");
    }
    return GM_OK;
}

extern "C" int gm_lbfgs_set_old(gm_lbfgs *h, const float *grad_old, const float *model_old) {
    if (!h || !grad_old || !model_old) return gm::fail(GM_ERROR_INVALID, "gm_lbfgs_set_old: bad argument");
    LB_CUDA(cudaSetDevice(h->device), "gm_lbfgs_set_old");
    const size_t nvec = h->nvec;
    int rc;
    for (int w = 0; w < 2; ++w) {
        if ((rc = stage(h, h->grid, w ? model_old : grad_old, nvec, "gm_lbfgs_set_old"))) return rc;
        gm::k_to_vec<<<blocks(nvec), TPB, 0, h->st>>>(h->grid, w ? h->old_model : h->old_grad, nvec, h->n, h->nx,
                                                        h->ny);
        gm::note_launch();
    }
    LB_CUDA(cudaStreamSynchronize(h->st), "gm_lbfgs_set_old");
    h->have_old = true;
    return GM_OK;
}

extern "C" int gm_mat_change(int device, int n, int mode, float eps_scale, float low, float up, const float *hgrad,
                             const float *model_old, float *model) {
    if (n <= 0 || !hgrad || !model_old || !model || (mode != 0 && mode != 1))
        return gm::fail(GM_ERROR_INVALID, "gm_mat_change: bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return gm::fail(GM_ERROR_CUDA, "gm_mat_change: bad device %d", device);
    const size_t bytes = (size_t)n * sizeof(float);
    float *dh = nullptr, *dold = nullptr;
    int rc = GM_OK;
    cudaError_t e = cudaMalloc(&dh, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&dold, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(dh, hgrad, bytes, cudaMemcpyDefault);
    if (e == cudaSuccess) e = cudaMemcpy(dold, model_old, bytes, cudaMemcpyDefault);
    if (e == cudaSuccess) {
        gm::k_mat_change<<<blocks(n), TPB>>>(dh, dold, dh, (size_t)n, eps_scale, low, up, mode);
        gm::note_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(model, dh, bytes, cudaMemcpyDefault);
    if (e != cudaSuccess) rc = cuda_fail(e, "gm_mat_change");
    cudaFree(dh);
    cudaFree(dold);
    return rc;
}
