// gm_solve_noalloc: the block solve + FP64 refinement of gm_solve without
// any device allocation.
//
// Who needs it: callers that cannot call cudaMalloc/cudaFree at solve time.
// cudaFree synchronises the whole device and cudaMalloc can, so a host code
// that keeps its own kernels running on other streams of the same GPU (for
// example a time-domain modelling job sharing the GPU with the
// frequency-domain engine) cannot let a solve stall them; and a caller that
// has reserved the device memory it may use up front (a fixed budget handed
// to its own pool allocator) has nothing left for us to allocate from.
// gm_solve grows its workspaces with cudaMalloc on first use; this entry
// point instead carves them out of one file-scope device array of fixed size
// (GM_NOALLOC_SCRATCH_BYTES below), so it serves small problems only and
// rejects larger ones with GM_ERROR_INVALID.
//
// The array is loaded on a device together with this file's module.  CUDA
// loads modules lazily (on first use), and loading one takes device memory,
// so gm_engine_create does that set-up once per device, with the device
// current: it looks the array's address up with cudaGetSymbolAddress and
// loads every substitution and refinement kernel the entry point launches
// (noalloc_prepare below).  From then on the array stays resident on that
// device until the process exits, and a gm_solve_noalloc call allocates
// nothing.  Every call shares the array and leaves its contents behind:
// nothing in it is read before this call writes it (the solution buffer,
// which the refinement accumulates into, is the caller's and is cleared
// first), and two calls whose GPU work overlaps -- from two threads, or two
// engines on different streams of the same device -- race on it.  The
// refinement loop reads the residual norms back to the host and waits for
// the engine's stream once per sweep.
#include <cmath>
#include <mutex>

#include "engine.hpp"

namespace {

constexpr size_t kScratchBytes = (size_t)32 << 20;   // GM_NOALLOC_SCRATCH_BYTES
constexpr int kMaxDevices = 64;
constexpr int kMaxNormPairs = 4096;                  // frequencies x right-hand sides

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices] = {};

// device address of the scratch array on `device` (which must be current)
int scratch_address(int device, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return gm::fail(GM_ERROR_INVALID, "gm_solve_noalloc: device index %d unsupported", device);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess || !p)
            return gm::fail(GM_ERROR_CUDA, "gm_solve_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(err));
        g_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_addr[device]);
    return GM_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// true when p is memory a kernel on the current device can use: device or
// managed memory (a host pointer would fault there, or on a system with
// heterogeneous memory access silently read host memory)
bool device_reachable(const void *p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();   // clear the error of an unknown pointer
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

template <class R>
void substitute_into(gm_engine *e, void *xT, void *w, int nrhs, int trans) {
    gm::SolveArgs<R> a{};
    a.s = e->dsym;
    a.front = e->d_front.p;
    a.pivsrc = e->cfg.pivot_tol > 0 ? e->d_pivsrc.as<unsigned char>() : nullptr;
    a.x = xT;
    a.w = w;
    a.nf = e->nf;
    a.nrhs = nrhs;
    a.ldr = nrhs;
    const int nchunk = (nrhs + 31) / 32;
    a.rch = (nrhs + nchunk - 1) / nchunk;
    a.trans = trans;
    for (int h = 0; h < (int)e->levels.size(); ++h) gm::launch_solve_forward_level<R>(a, e->levels[h], e->st);
    for (int h = (int)e->levels.size() - 1; h >= 0; --h) gm::launch_solve_backward_level<R>(a, e->levels[h], e->st);
}

}  // namespace

namespace gm {
// Once per device, with that device current (gm_engine_create): the scratch
// array's address and every kernel gm_solve_noalloc launches, so that the
// entry point itself never triggers a lazy module load.
int noalloc_prepare(int device) {
    unsigned char *base = nullptr;
    const int rc = scratch_address(device, &base);
    if (rc) return rc;
    (void)cudaGetLastError();   // an earlier call's error is not this load's
    preload_solve_kernels();
    preload_refine_kernels();
    preload_gmres_kernels();
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return fail(GM_ERROR_CUDA, "loading the solve kernels failed: %s", cudaGetErrorString(err));
    return GM_OK;
}
}  // namespace gm

#define NA_CUDA(call)                                                                                       \
    do {                                                                                                    \
        cudaError_t err_ = (call);                                                                          \
        if (err_ != cudaSuccess)                                                                            \
            return gm::fail(GM_ERROR_CUDA, "%s failed: %s", #call, cudaGetErrorString(err_));              \
    } while (0)

extern "C" int gm_solve_noalloc(gm_engine *e, int sys, int nrhs, const double *d_b, double *d_x) {
    if (!e || !d_b || !d_x || nrhs <= 0) return gm::fail(GM_ERROR_INVALID, "gm_solve_noalloc: bad argument");
    if (sys != GM_SYS_A && sys != GM_SYS_AT) return gm::fail(GM_ERROR_INVALID, "gm_solve_noalloc: unknown sys %d", sys);
    if (!e->factored) return gm::fail(GM_ERROR_STATE, "gm_solve_noalloc: no factorisation (gm_factor)");
    NA_CUDA(cudaSetDevice(e->device));

    const bool fp64 = e->cfg.precision == GM_PREC_FP64;
    const size_t cs = e->csize();
    const size_t cnt = (size_t)e->nf * e->n * nrhs;
    if (!device_reachable(d_b) || !device_reachable(d_x))
        return gm::fail(GM_ERROR_INVALID, "gm_solve_noalloc: b and x must be device (or managed) memory");
    {
        const uintptr_t b0 = (uintptr_t)d_b, x0 = (uintptr_t)d_x, nb = cnt * sizeof(double2);
        if (b0 < x0 + nb && x0 < b0 + nb)
            return gm::fail(GM_ERROR_INVALID, "gm_solve_noalloc: b and x overlap");
    }
    const int nblk = gm::residual_blocks(e->cfg.nx, e->cfg.ny);
    const int npairs = e->nf * nrhs;
    const size_t b_t = align256(cnt * cs);
    const size_t b_w = align256((size_t)e->nf * e->sym.rhs_total * nrhs * cs);
    const size_t b_r = align256(cnt * sizeof(double2));
    const size_t b_p = align256((size_t)nblk * npairs * 2 * sizeof(double));
    const size_t b_n = align256((size_t)npairs * 2 * sizeof(double));
    const size_t need = b_t + b_w + b_r + b_p + b_n;
    if (need > kScratchBytes || npairs > kMaxNormPairs)
        return gm::fail(GM_ERROR_INVALID,
                        "gm_solve_noalloc: %d frequencies x %d right-hand sides on %d unknowns need %zu bytes of "
                        "scratch; the fixed scratch array holds %zu bytes (use gm_solve)",
                        e->nf, nrhs, e->n, need, kScratchBytes);
    unsigned char *base = nullptr;
    int rc = scratch_address(e->device, &base);
    if (rc) return rc;
    void *t = base;
    void *w = base + b_t;
    double2 *r = reinterpret_cast<double2 *>(base + b_t + b_w);
    double *part = reinterpret_cast<double *>(base + b_t + b_w + b_r);
    double *norm = reinterpret_cast<double *>(base + b_t + b_w + b_r + b_p);
    const double2 *b = reinterpret_cast<const double2 *>(d_b);
    double2 *x = reinterpret_cast<double2 *>(d_x);

    // initial solve in working precision, x = 0 + t
    NA_CUDA(cudaEventRecord(e->ev0, e->st));
    if (fp64) gm::launch_convert_down<double>(b, t, cnt, e->st);
    else gm::launch_convert_down<float>(b, t, cnt, e->st);
    NA_CUDA(cudaMemsetAsync(x, 0, cnt * sizeof(double2), e->st));
    if (fp64) substitute_into<double>(e, t, w, nrhs, sys);
    else substitute_into<float>(e, t, w, nrhs, sys);
    if (fp64) gm::launch_add_up<double>(x, t, cnt, e->st);
    else gm::launch_add_up<float>(x, t, cnt, e->st);
    NA_CUDA(cudaGetLastError());
    NA_CUDA(cudaEventRecord(e->ev1, e->st));
    NA_CUDA(cudaEventSynchronize(e->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    e->stats.ms_solve = ms;
    e->stats.ms_refine = 0;
    e->stats.ms_subst = 0;       // substitutions are not timed separately here
    e->stats.ms_subst_bwd = 0;
    e->stats.n_subst = 1;
    NA_CUDA(cudaEventRecord(e->ev0, e->st));

    gm::ResidArgs ra{};
    ra.nx = e->cfg.nx; ra.ny = e->cfg.ny; ra.n = e->n; ra.nf = e->nf; ra.nrhs = nrhs; ra.ldr = nrhs;
    ra.A = e->d_A.as<double2>(); ra.x = x; ra.b = b; ra.r = r;
    ra.op_mode = e->cfg.op_mode; ra.trans = sys;
    static thread_local double h_norm[2 * kMaxNormPairs];
    double worst = 0;
    int it = 0;
    for (;; ++it) {
        const int used = gm::launch_residual(ra, part, nblk, e->st);
        gm::launch_reduce_norms(part, used, 2 * npairs, norm, e->st);
        NA_CUDA(cudaGetLastError());
        NA_CUDA(cudaMemcpyAsync(h_norm, norm, 2 * npairs * sizeof(double), cudaMemcpyDeviceToHost, e->st));
        NA_CUDA(cudaStreamSynchronize(e->st));
        worst = 0;
        bool finite = true;
        for (int c = 0; c < npairs; ++c) {
            const double rr = h_norm[2 * c], bb = h_norm[2 * c + 1];
            if (!std::isfinite(rr)) finite = false;
            const double rel = bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
            worst = rel > worst ? rel : worst;
        }
        if (!finite) {
            e->stats.ir_iterations = it;
            e->stats.ir_residual = NAN;
            return gm::fail(GM_ERROR_NONFINITE, "gm_solve_noalloc: non-finite residual after %d sweeps", it);
        }
        if (worst <= e->cfg.ir_tol || it >= e->cfg.ir_max_iter) break;
        if (fp64) gm::launch_convert_down<double>(r, t, cnt, e->st);
        else gm::launch_convert_down<float>(r, t, cnt, e->st);
        if (fp64) substitute_into<double>(e, t, w, nrhs, sys);
        else substitute_into<float>(e, t, w, nrhs, sys);
        if (fp64) gm::launch_add_up<double>(x, t, cnt, e->st);
        else gm::launch_add_up<float>(x, t, cnt, e->st);
        e->stats.n_subst += 1;
    }
    NA_CUDA(cudaEventRecord(e->ev1, e->st));
    NA_CUDA(cudaEventSynchronize(e->ev1));
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    e->stats.ms_refine = ms;
    e->stats.ir_iterations = it;
    e->stats.ir_residual = worst;
    return worst <= e->cfg.ir_tol ? GM_OK : GM_WARNING_NOT_CONVERGED;
}
