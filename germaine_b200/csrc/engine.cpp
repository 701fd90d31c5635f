// gm_engine: the C-ABI of the per-frequency engine (include/germaine_gpu.h).
//
// Memory plan (HBM, per engine):
//   symbolic structure        ~ 40 B per grid point (uploaded once)
//   A      [nf][9][n] c128    assembled stencils of the frequency batch
//   fronts [nf][sum f^2]      c128 (GM_PREC_FP64) or c64 (GM_PREC_C64_IR)
//   x, b, r[nf][n][nrhs] c128 solution, right-hand side, residual
//   t      [nf][n][nrhs]      working precision copy for the substitution
//   w      [nf][sum f][nrhs]  front-vector workspace of the substitution
// At 841 x 227 (n = 190,907) with 10 frequencies x 100 shots this is about
// 8 GB of fronts in FP64 plus 12 GB of vectors -- resident in one B200.
#include "engine.hpp"
#include "kernels_epi.cuh"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>

#include "host_setup.h"
#include "kernels_tc.cuh"

using gm::fail;

#define GM_CUDA(call)                                                                                       \
    do {                                                                                                    \
        cudaError_t err_ = (call);                                                                          \
        if (err_ != cudaSuccess)                                                                            \
            return fail(GM_ERROR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_), __FILE__, \
                        __LINE__);                                                                          \
    } while (0)

#define GM_ALLOC(buf, nbytes)                                                                                   \
    do {                                                                                                        \
        cudaError_t err_ = (buf).ensure(nbytes);                                                                \
        if (err_ != cudaSuccess)                                                                                \
            return fail(err_ == cudaErrorMemoryAllocation ? GM_ERROR_OUT_OF_MEMORY : GM_ERROR_CUDA,             \
                        "device allocation of %zu bytes failed: %s", (size_t)(nbytes), cudaGetErrorString(err_)); \
    } while (0)

namespace {

template <class T>
int upload(gm::DevBuf &buf, const std::vector<T> &v, cudaStream_t st) {
    GM_ALLOC(buf, v.size() * sizeof(T));
    if (!v.empty()) GM_CUDA(cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return GM_OK;
}

int check_config(const gm_config *c) {
    if (!c) return fail(GM_ERROR_INVALID, "null config");
    if (c->nx < 3 || c->ny < 3) return fail(GM_ERROR_INVALID, "grid must be at least 3 x 3 (got %d x %d)", c->nx, c->ny);
    if ((int64_t)c->nx * c->ny > (int64_t)1 << 27) return fail(GM_ERROR_INVALID, "grid too large");
    if (!(c->dh > 0.f)) return fail(GM_ERROR_INVALID, "DH must be positive");
    if (c->npml < 0 || 2 * c->npml >= c->nx || 2 * c->npml >= c->ny)
        return fail(GM_ERROR_INVALID, "NPML %d does not fit the %d x %d grid", c->npml, c->nx, c->ny);
    if (c->physics != GM_PHYS_AC && c->physics != GM_PHYS_SH && c->physics != GM_PHYS_TE)
        return fail(GM_ERROR_INVALID, "unknown physics %d", c->physics);
    if (c->precision != GM_PREC_FP64 && c->precision != GM_PREC_C64_IR)
        return fail(GM_ERROR_INVALID, "unknown precision %d", c->precision);
    if (c->op_mode != GM_OP_REF && c->op_mode != GM_OP_EXACT) return fail(GM_ERROR_INVALID, "unknown op_mode %d", c->op_mode);
    if (c->refine < GM_REFINE_MODE_AUTO || c->refine > GM_REFINE_MODE_GMRES)
        return fail(GM_ERROR_INVALID, "unknown refinement mode %d", c->refine);
    if (c->gmres_restart < 0) return fail(GM_ERROR_INVALID, "GMRES restart length must be >= 0");
    return GM_OK;
}

}  // namespace

extern "C" int gm_engine_create(int device, const gm_config *cfg, gm_engine **out) {
    if (!out) return fail(GM_ERROR_INVALID, "gm_engine_create: null output");
    *out = nullptr;
    int rc = check_config(cfg);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(GM_ERROR_CUDA, "no CUDA device available: the engine has no CPU path");
    if (device < 0 || device >= ndev) return fail(GM_ERROR_INVALID, "device %d out of range (%d devices)", device, ndev);
    GM_CUDA(cudaSetDevice(device));

    gm_engine *e = nullptr;
    try {
        e = new gm_engine();
        e->cfg = *cfg;
        if (e->cfg.leaf_max <= 0) e->cfg.leaf_max = 32;   // measured best at 841 x 227 (24 .. 40 within 6 %)
        if (!(e->cfg.ir_tol > 0)) e->cfg.ir_tol = 1e-10;
        if (e->cfg.pivot_tol == 0) e->cfg.pivot_tol = 0.1;
        if (e->cfg.ir_max_iter <= 0) e->cfg.ir_max_iter = 10;
        if (e->cfg.gmres_restart <= 0 || e->cfg.gmres_restart > gm::kGmresMaxRestart)
            e->cfg.gmres_restart = gm::kGmresMaxRestart;
        e->device = device;
        e->fsshift = cfg->free_surf ? 0 : cfg->npml;
        e->n = cfg->nx * cfg->ny;
        gm::build_symbolic(cfg->nx, cfg->ny, e->cfg.leaf_max, e->sym);
    } catch (const std::bad_alloc &) {
        delete e;
        return fail(GM_ERROR_OUT_OF_MEMORY, "host allocation failed in gm_engine_create");
    } catch (const std::exception &ex) {
        delete e;
        return fail(GM_ERROR_INVALID, "symbolic analysis failed: %s", ex.what());
    }
    std::unique_ptr<gm_engine> guard(e);
    GM_CUDA(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
    GM_CUDA(cudaEventCreate(&e->ev0));
    GM_CUDA(cudaEventCreate(&e->ev1));
    GM_CUDA(cudaEventCreate(&e->ev_s0));
    GM_CUDA(cudaEventCreate(&e->ev_s1));
    GM_CUDA(cudaEventCreate(&e->ev_sm));
    if ((rc = gm::noalloc_prepare(device))) return rc;

    const gm::Symbolic &s = e->sym;
    // level-ordered entry lists in the configured operator orientation
    std::vector<int64_t> ent_dst;
    std::vector<int> ent_src;
    std::vector<int64_t> ent_lvl_off(s.nnodes + 1, 0);
    ent_dst.reserve(s.ent_pos.size());
    ent_src.reserve(s.ent_pos.size());
    e->levels.resize(s.nlevels);
    for (int h = 0; h < s.nlevels; ++h) {
        gm::LevelInfo &L = e->levels[h];
        L.index = h;
        L.first = s.lvl_off[h];
        L.count = s.lvl_off[h + 1] - s.lvl_off[h];
        L.max_front = s.lvl_max_front[h];
        L.max_piv = s.lvl_max_piv[h];
        L.max_ring = 0;
        L.mid_words = 0;
        for (int t = L.first; t < L.first + L.count; ++t) {
            const int v = s.lvl_nodes[t], fv = s.nfront[v], sv = s.npiv[v];
            L.max_ring = std::max(L.max_ring, fv - sv);
            L.mid_words = std::max(L.mid_words, (int64_t)(fv + 1) * sv + (int64_t)(sv | 1) * (fv - sv));
        }
        L.ent_first = (int64_t)ent_dst.size();
        for (int t = L.first; t < L.first + L.count; ++t) {
            const int v = s.lvl_nodes[t];
            ent_lvl_off[t] = (int64_t)ent_dst.size();
            for (int64_t q = s.ent_off[v]; q < s.ent_off[v + 1]; ++q) {
                ent_dst.push_back(s.front_off[v] + s.ent_pos[q]);
                int id = s.ent_id[q];
                if (e->cfg.op_mode == GM_OP_EXACT) {   // M = A: entry (r, c) reads A[r][c]
                    const int dir = id / s.n, c = id % s.n;
                    const int r = c + gm::stencil_di(dir) + gm::stencil_dj(dir) * s.nx;
                    id = (8 - dir) * s.n + r;
                }
                ent_src.push_back(id);
            }
        }
        L.ent_count = (int64_t)ent_dst.size() - L.ent_first;
    }
    ent_lvl_off[s.nnodes] = (int64_t)ent_dst.size();
    int rc2;
    if ((rc2 = upload(e->d_npiv, s.npiv, e->st)) || (rc2 = upload(e->d_nfront, s.nfront, e->st)) ||
        (rc2 = upload(e->d_child0, s.child0, e->st)) || (rc2 = upload(e->d_child1, s.child1, e->st)) ||
        (rc2 = upload(e->d_vars, s.vars, e->st)) || (rc2 = upload(e->d_inv, s.inv, e->st)) ||
        (rc2 = upload(e->d_lvl_nodes, s.lvl_nodes, e->st)) || (rc2 = upload(e->d_front_off, s.front_off, e->st)) ||
        (rc2 = upload(e->d_var_off, s.var_off, e->st)) || (rc2 = upload(e->d_inv_off, s.inv_off, e->st)) ||
        (rc2 = upload(e->d_rhs_off, s.rhs_off, e->st)) || (rc2 = upload(e->d_ent_dst, ent_dst, e->st)) ||
        (rc2 = upload(e->d_ent_src, ent_src, e->st)) || (rc2 = upload(e->d_ent_lvl_off, ent_lvl_off, e->st)))
        return rc2;
    GM_CUDA(cudaStreamSynchronize(e->st));
    gm::DevSym &d = e->dsym;
    d.n = s.n; d.nnodes = s.nnodes;
    d.npiv = e->d_npiv.as<int>(); d.nfront = e->d_nfront.as<int>();
    d.child0 = e->d_child0.as<int>(); d.child1 = e->d_child1.as<int>();
    d.vars = e->d_vars.as<int>(); d.inv = e->d_inv.as<int>(); d.lvl_nodes = e->d_lvl_nodes.as<int>();
    d.front_off = e->d_front_off.as<int64_t>(); d.var_off = e->d_var_off.as<int64_t>();
    d.inv_off = e->d_inv_off.as<int64_t>(); d.rhs_off = e->d_rhs_off.as<int64_t>();
    d.front_total = s.front_total; d.rhs_total = s.rhs_total;

    gm_stats &st = e->stats;
    st.n = s.n;
    st.nonzero = 9LL * cfg->nx * cfg->ny - 6LL * cfg->nx - 6LL * cfg->ny + 4;
    st.nnodes = s.nnodes; st.nlevels = s.nlevels;
    st.max_front = *std::max_element(s.nfront.begin(), s.nfront.end());
    st.max_piv = *std::max_element(s.npiv.begin(), s.npiv.end());
    st.front_entries = s.front_total;
    st.factor_entries = s.factor_entries;
    st.u_entries = s.u_entries;
    st.factor_flops = s.factor_flops;
    st.solve_flops_per_rhs = s.solve_flops_per_rhs;
    *out = guard.release();
    return GM_OK;
}

extern "C" int gm_engine_destroy(gm_engine *e) {
    if (!e) return GM_OK;
    cudaSetDevice(e->device);
    if (e->st) cudaStreamSynchronize(e->st);
    delete e;  // releases the stream, the events and every device buffer
    return GM_OK;
}

extern "C" int gm_engine_stats(const gm_engine *e, gm_stats *out) {
    if (!e || !out) return fail(GM_ERROR_INVALID, "gm_engine_stats: null argument");
    *out = e->stats;
    out->kernel_launches = gm::launch_count();
    return GM_OK;
}

extern "C" int gm_engine_stream(const gm_engine *e, void **stream) {
    if (!e || !stream) return fail(GM_ERROR_INVALID, "gm_engine_stream: null argument");
    *stream = (void *)e->st;
    return GM_OK;
}

extern "C" int gm_set_models(gm_engine *e, int nmod, const float *mat0, const float *mat1) {
    if (!e || nmod <= 0 || !mat0 || !mat1) return fail(GM_ERROR_INVALID, "gm_set_models: bad argument");
    GM_CUDA(cudaSetDevice(e->device));
    const size_t nb = (size_t)nmod * e->n * sizeof(float);
    GM_ALLOC(e->d_m0, nb);
    GM_ALLOC(e->d_m1, nb);
    GM_CUDA(cudaMemcpyAsync(e->d_m0.p, mat0, nb, cudaMemcpyDefault, e->st));
    GM_CUDA(cudaMemcpyAsync(e->d_m1.p, mat1, nb, cudaMemcpyDefault, e->st));
    GM_CUDA(cudaStreamSynchronize(e->st));
    e->nmod = nmod;
    e->have_model = true;
    e->factored = false;
    return GM_OK;
}

extern "C" int gm_set_model(gm_engine *e, const float *mat0, const float *mat1) {
    if (!e || !mat0 || !mat1) return fail(GM_ERROR_INVALID, "gm_set_model: null argument");
    return gm_set_models(e, 1, mat0, mat1);
}

namespace gm {

// Assemble all frequencies of the batch into e->d_A (device, asynchronous).
static int assemble_batch(gm_engine *e) {
    const gm_config &c = e->cfg;
    const int n = e->n, nf = e->nf;
    const int pml_stride = 4 * (c.nx + 2) + 4 * (c.ny + 2);
    std::vector<float> pml((size_t)nf * pml_stride);
    std::vector<AsmFreq> fq(nf);
    for (int f = 0; f < nf; ++f) {
        gmh_pml(c.nx, c.ny, c.dh, c.npml, c.free_surf, c.a0_pml, c.s, e->freqs[f], pml.data() + (size_t)f * pml_stride);
        float om2[2], om[2], om2mu0[2];
        gmh_assembly_scalars(c.physics, e->freqs[f], c.s, om2, om, om2mu0);
        fq[f].om2 = make_float2(om2[0], om2[1]);
        fq[f].om = make_float2(om[0], om[1]);
        fq[f].om2mu0 = make_float2(om2mu0[0], om2mu0[1]);
        fq[f].model = e->models[f];
        fq[f].pad = 0;
    }
    GM_ALLOC(e->d_A, (size_t)nf * 9 * n * sizeof(double2));
    GM_ALLOC(e->d_mass, (size_t)nf * n * sizeof(float2));
    GM_ALLOC(e->d_stiff, (size_t)nf * n * sizeof(float));
    GM_ALLOC(e->d_pml, pml.size() * sizeof(float));
    GM_ALLOC(e->d_fq, fq.size() * sizeof(AsmFreq));
    GM_CUDA(cudaMemcpyAsync(e->d_pml.p, pml.data(), pml.size() * sizeof(float), cudaMemcpyHostToDevice, e->st));
    GM_CUDA(cudaMemcpyAsync(e->d_fq.p, fq.data(), fq.size() * sizeof(AsmFreq), cudaMemcpyHostToDevice, e->st));
    AsmArgs a{};
    a.nx = c.nx; a.ny = c.ny; a.n = n; a.nf = nf; a.physics = c.physics;
    gmh_fd_weights(c.dh, a.w);
    a.pml = e->d_pml.as<float>();
    a.pml_stride = pml_stride;
    a.stiff = e->d_stiff.as<float>();
    a.mass = e->d_mass.as<float2>();
    a.A = e->d_A.as<double2>();
    launch_assemble(a, e->d_m0.as<float>(), e->d_m1.as<float>(), e->d_fq.as<AsmFreq>(), e->d_stiff.as<float>(), e->st);
    GM_CUDA(cudaGetLastError());
    return GM_OK;
}

// Builds the per-level list of contribution-block products
// C[s:f, s:f] -= L21 * U12 (K = npiv) over every front and frequency, and
// their output tiles: tcgen05 tiles (128 x 64) for the complex64 path on
// levels whose blocks are large enough to fill them, CUDA-core tiles
// (64 x 64) otherwise.
// Levels of fronts with at most 16 pivots that are too large for the small
// kernel go to the fused mid-level kernel; GM_NO_FACTOR_MID=1 keeps them on
// the blocked diagonal / panel / contribution-GEMM sequence.  With 17-32
// pivots the fused kernel holds 32-entry pivot rows in registers and fits
// one CTA per SM; measured at 841 x 227 (10 frequencies) the blocked
// sequence is faster there (levels 5-6, 26-28 pivots: 1.64 -> 1.26 and
// 1.22 -> 1.10 ms) and slower with 14 pivots (level 4: 1.05 vs 1.39 ms).
// GM_MID_MAX_PIV=<n> moves the limit (32: every level the kernel takes).
template <class R>
static bool use_mid_factor(const LevelInfo &L) {
    static const bool off = std::getenv("GM_NO_FACTOR_MID") != nullptr;
    static const int max_piv = [] {
        const char *v = std::getenv("GM_MID_MAX_PIV");
        return v ? std::atoi(v) : 16;
    }();
    return !off && L.max_piv <= max_piv && mid_factor_level<R>(L);
}

template <class R>
static int build_cb_plan(gm_engine *e) {
    using C = cplx_any<R>;
    const Symbolic &s = e->sym;
    const bool c64 = e->cfg.precision == GM_PREC_C64_IR;
    // Smallest contribution block routed to the tcgen05 kernel
    // (gm_config.tc_min_block; GM_TC_MIN_BLOCK=<rows> overrides it).  Off by
    // default: measured on 841 x 227 with 10 frequencies x 100 shots, routing
    // the blocks of >= 128 rows makes the complex64 factorisation slower
    // (14.72 vs 14.24 ms: the kernel keeps its tensor pipe 15-20 % busy) and
    // its truncating accumulation costs the 3 Hz matrix a fourth sweep
    // (92.5 -> 110 ms per step), while the block GEMM is ~1.4 % of the GPU
    // time of a step.
    int kTcMinBlock = e->cfg.tc_min_block > 0 ? e->cfg.tc_min_block : 1 << 30;
    if (const char *v = std::getenv("GM_TC_MIN_BLOCK")) kTcMinBlock = std::atoi(v);
    std::vector<GemmProb<R>> probs;
    std::vector<int4> tiles;
    e->stats.tc_tiles = 0;
    e->cb_plan.assign(e->levels.size(), {});
    C *base = e->d_front.as<C>();
    for (size_t h = 0; h < e->levels.size(); ++h) {
        const LevelInfo &L = e->levels[h];
        int max_cb = 0;
        for (int t = L.first; t < L.first + L.count; ++t) {
            const int v = s.lvl_nodes[t];
            max_cb = std::max(max_cb, s.nfront[v] - s.npiv[v]);
        }
        const int backend = (c64 && max_cb >= kTcMinBlock) ? 1 : 0;
        const int tr = backend ? cgemm_tile_rows() : kGemmTileCC, tc = backend ? cgemm_tile_cols() : kGemmTileCC;
        auto &pl = e->cb_plan[h];
        pl.backend = backend;
        pl.prob_off = (int64_t)probs.size();
        pl.tile_off = (int64_t)tiles.size();
        if (small_factor_level<R>(L) || use_mid_factor<R>(L)) {   // fused kernels form the Schur complement themselves
            pl.ntiles = 0;
            continue;
        }
        for (int f = 0; f < e->nf; ++f)
            for (int t = L.first; t < L.first + L.count; ++t) {
                const int v = s.lvl_nodes[t];
                const int fr = s.nfront[v], sp = s.npiv[v], m = fr - sp;
                if (sp == 0 || m == 0) continue;
                C *F = base + (size_t)f * s.front_total + s.front_off[v];
                GemmProb<R> p{F + sp, F + (size_t)sp * fr, F + sp + (size_t)sp * fr, fr, fr, fr, m, m, sp};
                const int id = (int)(probs.size() - pl.prob_off);
                probs.push_back(p);
                for (int a = 0; a < (m + tr - 1) / tr; ++a)
                    for (int b = 0; b < (m + tc - 1) / tc; ++b) tiles.push_back(make_int4(id, a, b, 0));
            }
        pl.ntiles = (int)(tiles.size() - pl.tile_off);
        if (backend == 1) e->stats.tc_tiles += pl.ntiles;
    }
    GM_ALLOC(e->d_cb_probs, probs.size() * sizeof(GemmProb<R>) + 16);
    GM_ALLOC(e->d_cb_tiles, tiles.size() * sizeof(int4) + 16);
    GM_ALLOC(e->d_tcerr, sizeof(int));
    if (!probs.empty())
        GM_CUDA(cudaMemcpyAsync(e->d_cb_probs.p, probs.data(), probs.size() * sizeof(GemmProb<R>), cudaMemcpyHostToDevice, e->st));
    if (!tiles.empty())
        GM_CUDA(cudaMemcpyAsync(e->d_cb_tiles.p, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice, e->st));
    GM_CUDA(cudaStreamSynchronize(e->st));
    e->cb_plan_base = e->d_front.p;
    e->cb_plan_nf = e->nf;
    return GM_OK;
}

template <class R>
static int factor_batch(gm_engine *e, double pivscale) {
    FactorArgs<R> a{};
    a.s = e->dsym;
    a.front = e->d_front.p;
    a.A = e->d_A.as<double2>();
    a.ent_dst = e->d_ent_dst.as<int64_t>();
    a.ent_src = e->d_ent_src.as<int>();
    a.ent_lvl_off = e->d_ent_lvl_off.as<int64_t>();
    a.nf = e->nf;
    a.amax = e->d_amax.as<unsigned long long>();
    a.pivscale = pivscale;
    a.npert = e->d_npert.as<unsigned long long>();
    a.nswap = a.npert + 1;
    a.pivtau2 = e->cfg.pivot_tol > 0 ? e->cfg.pivot_tol * e->cfg.pivot_tol : 0.0;
    a.pivsrc = e->cfg.pivot_tol > 0 ? e->d_pivsrc.as<unsigned char>() : nullptr;
    if (e->cb_plan_base != e->d_front.p || e->cb_plan_nf != e->nf) {
        const int rc = build_cb_plan<R>(e);
        if (rc) return rc;
    }
    GM_CUDA(cudaMemsetAsync(e->d_tcerr.p, 0, sizeof(int), e->st));
    const GemmProb<R> *probs = e->d_cb_probs.as<GemmProb<R>>();
    const int4 *tiles = e->d_cb_tiles.as<int4>();
    // GM_TRACE_LEVELS=1: device time of every level on stderr
    static const bool trace = std::getenv("GM_TRACE_LEVELS") != nullptr;
    static const bool no_graph = std::getenv("GM_NO_GRAPH") != nullptr;
    const int nl = (int)e->levels.size();
    auto launch_levels = [&](cudaEvent_t *evs) {
        for (int h = 0; h < nl; ++h) {
            if (small_factor_level<R>(e->levels[h])) {
                launch_factor_small<R>(a, e->levels[h], e->st);
            } else if (use_mid_factor<R>(e->levels[h])) {
                launch_factor_mid<R>(a, e->levels[h], e->st);
            } else {
                launch_factor_level<R>(a, e->levels[h], e->st);
                const auto &pl = e->cb_plan[h];
                if (pl.backend == 1)
                    launch_cgemm_sub(1, reinterpret_cast<const CgemmProb *>(probs + pl.prob_off), tiles + pl.tile_off,
                                     pl.ntiles, e->d_tcerr.as<int>(), e->st);
                else
                    launch_gemm_sub_cc<R>(probs + pl.prob_off, tiles + pl.tile_off, pl.ntiles, e->st);
            }
            if (evs) cudaEventRecord(evs[1 + h], e->st);
        }
    };
    if (!trace && !no_graph && !e->fgraph_broken) {
        // every level of the factorisation as one CUDA graph, replayed while
        // the buffers and the batch stay the same.  The first factorisation
        // with new buffers launches directly (which also sets every kernel's
        // attributes outside any capture), the second captures the graph.
        gm_engine::FactorGraphKey key;
        key.front = e->d_front.p; key.A = e->d_A.p; key.amax = e->d_amax.p; key.npert = e->d_npert.p;
        key.pivsrc = e->d_pivsrc.p;
        key.tcerr = e->d_tcerr.p; key.probs = probs; key.tiles = tiles; key.nf = e->nf; key.fp64 = sizeof(R) == 8;
        if (!(e->fgraph && key == e->fgraph_key) && key == e->fgraph_seen) {
            if (e->fgraph) cudaGraphExecDestroy(e->fgraph);
            e->fgraph = nullptr;
            cudaGraph_t g = nullptr;
            const long long before = launch_count();
            bool ok = cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                launch_levels(nullptr);
                ok = cudaStreamEndCapture(e->st, &g) == cudaSuccess && g;
            }
            if (ok) ok = cudaGraphInstantiate(&e->fgraph, g, 0) == cudaSuccess;
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();   // a failed capture leaves its error here
            if (ok) {
                e->fgraph_key = key;
                e->fgraph_kernels = launch_count() - before;
            } else {
                e->fgraph = nullptr;
                e->fgraph_broken = true;   // launch directly from now on
            }
        }
        e->fgraph_seen = key;
        if (e->fgraph && key == e->fgraph_key) {
            GM_CUDA(cudaGraphLaunch(e->fgraph, e->st));
            note_launches(e->fgraph_kernels);
            GM_CUDA(cudaGetLastError());
            return GM_OK;
        }
    }
    std::vector<cudaEvent_t> ev;
    if (trace) {
        ev.resize(nl + 1);
        for (auto &x : ev) cudaEventCreate(&x);
        cudaEventRecord(ev[0], e->st);
    }
    launch_levels(trace ? ev.data() : nullptr);
    if (trace) {
        cudaEventSynchronize(ev[nl]);
        for (int h = 0; h < nl; ++h) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev[h], ev[1 + h]);
            const LevelInfo &L = e->levels[h];
            std::fprintf(stderr, "factor %s level %2d: fronts %5d max_front %4d max_piv %4d %s %.3f ms\n",
                         sizeof(R) == 8 ? "c128" : "c64", h, L.count, L.max_front, L.max_piv,
                         small_factor_level<R>(L) ? "small" : use_mid_factor<R>(L) ? "mid" : "tiled", ms);
        }
        for (auto &x : ev) cudaEventDestroy(x);
    }
    GM_CUDA(cudaGetLastError());
    return GM_OK;
}

}  // namespace gm

namespace gm {

// The threshold-pivoting record starts as the identity: pivot k of a front
// takes row k % 32 of its 32-pivot block.  The factorisation rewrites the
// entries of the pivoted levels each time and never touches the others, so
// a slot is initialised once per buffer.
static int init_pivsrc(gm_engine *e) {
    if (e->pivsrc_ready != e->d_pivsrc.p) {
        e->pivsrc_ready = e->d_pivsrc.p;
        e->pivsrc_ready_nf = 0;
    }
    if (e->pivsrc_ready_nf >= e->nf) return GM_OK;
    const gm::Symbolic &s = e->sym;
    std::vector<unsigned char> ident((size_t)e->n, 0);
    for (int v = 0; v < s.nnodes; ++v)
        for (int k = 0; k < s.npiv[v]; ++k) ident[s.vars[s.var_off[v] + k]] = (unsigned char)(k % 32);
    for (int f = e->pivsrc_ready_nf; f < e->nf; ++f)
        GM_CUDA(cudaMemcpyAsync(e->d_pivsrc.as<unsigned char>() + (size_t)f * e->n, ident.data(), e->n,
                                cudaMemcpyHostToDevice, e->st));
    GM_CUDA(cudaStreamSynchronize(e->st));   // the host vector goes out of scope
    e->pivsrc_ready_nf = e->nf;
    return GM_OK;
}

// Numeric factorisation of the nf operators in e->d_A (assembled or given
// by value).  The static-pivot threshold is relative to max |A| over the
// whole batch, reduced on the device.
static int factor_assembled(gm_engine *e) {
    const bool fp64 = e->cfg.precision == GM_PREC_FP64;
    const size_t fbytes = (size_t)e->nf * e->sym.front_total * e->csize();
    GM_ALLOC(e->d_front, fbytes);
    GM_ALLOC(e->d_npert, 2 * sizeof(unsigned long long));   // perturbed pivots, row exchanges
    GM_ALLOC(e->d_amax, sizeof(unsigned long long));
    if (e->cfg.pivot_tol > 0) {
        GM_ALLOC(e->d_pivsrc, (size_t)e->nf * e->n);
        const int rc = init_pivsrc(e);
        if (rc) return rc;
    }
    GM_CUDA(cudaEventRecord(e->ev0, e->st));
    GM_CUDA(cudaMemsetAsync(e->d_npert.p, 0, 2 * sizeof(unsigned long long), e->st));
    GM_CUDA(cudaMemsetAsync(e->d_amax.p, 0, sizeof(unsigned long long), e->st));
    launch_amax(e->d_A.as<double2>(), (size_t)e->nf * 9 * e->n, e->d_amax.as<unsigned long long>(), e->st);
    const int rc = fp64 ? factor_batch<double>(e, 1e-13) : factor_batch<float>(e, 1e-6);
    if (rc) return rc;
    GM_CUDA(cudaEventRecord(e->ev1, e->st));
    GM_CUDA(cudaEventSynchronize(e->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    e->stats.ms_factor = ms;
    unsigned long long np = 0, amax_bits = 0, nsw = 0;
    GM_CUDA(cudaMemcpy(&np, e->d_npert.p, sizeof np, cudaMemcpyDeviceToHost));
    GM_CUDA(cudaMemcpy(&nsw, e->d_npert.as<unsigned long long>() + 1, sizeof nsw, cudaMemcpyDeviceToHost));
    e->stats.pivot_swaps = (int64_t)nsw;
    GM_CUDA(cudaMemcpy(&amax_bits, e->d_amax.p, sizeof amax_bits, cudaMemcpyDeviceToHost));
    double amax = 0;
    std::memcpy(&amax, &amax_bits, sizeof amax);
    if (!std::isfinite(amax))   // NaN bits order above every finite value in the max reduction
        return fail(GM_ERROR_NONFINITE, "factor: the operator holds non-finite values (NaN or Inf material?)");
    int tcerr = 0;
    GM_CUDA(cudaMemcpy(&tcerr, e->d_tcerr.p, sizeof tcerr, cudaMemcpyDeviceToHost));
    if (tcerr) return fail(GM_ERROR_CUDA, "factor: a tensor-core wait timed out in the contribution-block update");
    e->stats.perturbed_pivots = (int64_t)np;
    e->factored = true;
    return np ? GM_WARNING_PERTURBED : GM_OK;
}

}  // namespace gm

extern "C" int gm_factor_models(gm_engine *e, int nmat, const float *h_freqs, const int32_t *h_models) {
    if (!e || nmat <= 0 || !h_freqs) return fail(GM_ERROR_INVALID, "gm_factor: bad argument");
    if (!e->have_model) return fail(GM_ERROR_STATE, "gm_factor: no model set (gm_set_model)");
    for (int f = 0; f < nmat; ++f) {
        if (!(h_freqs[f] > 0.f) || !std::isfinite(h_freqs[f])) return fail(GM_ERROR_INVALID, "frequency %d is not positive", f);
        if (h_models && (h_models[f] < 0 || h_models[f] >= e->nmod))
            return fail(GM_ERROR_INVALID, "matrix %d: model %d out of range (%d models)", f, h_models[f], e->nmod);
    }
    GM_CUDA(cudaSetDevice(e->device));
    e->factored = false;
    e->values_only = false;
    e->nf = nmat;
    e->freqs.assign(h_freqs, h_freqs + nmat);
    if (h_models) e->models.assign(h_models, h_models + nmat);
    else e->models.assign(nmat, 0);

    GM_CUDA(cudaEventRecord(e->ev0, e->st));
    int rc = gm::assemble_batch(e);
    if (rc) return rc;
    GM_CUDA(cudaEventRecord(e->ev1, e->st));
    GM_CUDA(cudaEventSynchronize(e->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    e->stats.ms_assemble = ms;
    return gm::factor_assembled(e);
}

extern "C" int gm_factor(gm_engine *e, int nfreq, const float *h_freqs) {
    return gm_factor_models(e, nfreq, h_freqs, nullptr);
}

extern "C" int gm_factor_values(gm_engine *e, int nmat, const double *re, const double *im) {
    if (!e || nmat <= 0 || !re || !im) return fail(GM_ERROR_INVALID, "gm_factor_values: bad argument");
    GM_CUDA(cudaSetDevice(e->device));
    e->factored = false;
    e->values_only = true;
    e->nf = nmat;
    e->freqs.assign(nmat, 0.f);
    e->models.assign(nmat, 0);
    const size_t cnt = (size_t)nmat * 9 * e->n;
    GM_ALLOC(e->d_A, cnt * sizeof(double2));
    // split inputs staged in the (grow-only) residual workspace
    GM_ALLOC(e->d_r, 2 * cnt * sizeof(double));
    double *dre = e->d_r.as<double>(), *dim = dre + cnt;
    GM_CUDA(cudaEventRecord(e->ev0, e->st));
    GM_CUDA(cudaMemcpyAsync(dre, re, cnt * sizeof(double), cudaMemcpyDefault, e->st));
    GM_CUDA(cudaMemcpyAsync(dim, im, cnt * sizeof(double), cudaMemcpyDefault, e->st));
    gm::launch_pack_split(e->d_A.as<double2>(), dre, dim, cnt, e->st);
    GM_CUDA(cudaEventRecord(e->ev1, e->st));
    GM_CUDA(cudaEventSynchronize(e->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    e->stats.ms_assemble = ms;
    return gm::factor_assembled(e);
}

extern "C" int gm_get_triplets(gm_engine *e, int ifreq, double *Ar, double *Ai, int32_t *irow, int32_t *icol) {
    if (!e || ifreq < 0 || ifreq >= e->nf || !e->d_A.p) return fail(GM_ERROR_STATE, "gm_get_triplets: no assembled frequency %d", ifreq);
    GM_CUDA(cudaSetDevice(e->device));
    const int n = e->n, nx = e->cfg.nx, ny = e->cfg.ny;
    std::vector<double2> h((size_t)9 * n);
    GM_CUDA(cudaMemcpy(h.data(), e->d_A.as<double2>() + (size_t)ifreq * 9 * n, h.size() * sizeof(double2),
                       cudaMemcpyDeviceToHost));
    size_t c = 0;
    for (int k = 0; k < n; ++k) {
        const int x = k % nx, y = k / nx;
        for (int q = 0; q < 9; ++q) {
            const int xx = x + gm::stencil_di(q), yy = y + gm::stencil_dj(q);
            if (xx < 0 || xx >= nx || yy < 0 || yy >= ny) continue;
            const double2 v = h[(size_t)q * n + k];
            if (Ar) Ar[c] = v.x;
            if (Ai) Ai[c] = v.y;
            if (irow) irow[c] = k;
            if (icol) icol[c] = yy * nx + xx;
            ++c;
        }
    }
    return GM_OK;
}

namespace gm {

// One substitution over the right-hand sides in xT; fmap (device, nfz
// entries) restricts it to those matrices of the batch (NULL: all).
template <class R>
static void substitute(gm_engine *e, void *xT, int nrhs, int trans, const unsigned char *mask = nullptr,
                       const int *fmap = nullptr, int nfz = 0, const int *xmap = nullptr,
                       const SpikeRhs *spikes = nullptr) {
    cudaEventRecord(e->ev_s0, e->st);
    SolveArgs<R> a{};
    a.s = e->dsym;
    a.front = e->d_front.p;
    a.pivsrc = e->cfg.pivot_tol > 0 ? e->d_pivsrc.as<unsigned char>() : nullptr;
    a.x = xT;
    a.w = e->d_w.p;
    a.nf = e->nf;
    a.fmap = fmap;
    a.nfz = nfz;
    a.xmap = xmap;
    if (!e->lvl_cfg.empty() && e->tuned_nrhs == nrhs) a.lvl_cfg = e->lvl_cfg.data();
    if (mask && e->have_work) {   // the pruned pass launches only the live pairs
        a.work = e->d_work.as<int2>();
        a.work_off = e->work_off.data();
        a.work_w = e->work_w.data();
    }
    a.nrhs = nrhs;
    a.ldr = nrhs;
    const int nchunk = (nrhs + 31) / 32;
    a.rch = (nrhs + nchunk - 1) / nchunk;
    a.trans = trans;
    a.mask = mask;
    a.mask_nch = (nrhs + 31) / 32;
    if (spikes && mask) {   // implicit right-hand sides: x not cleared beforehand
        a.spike_k = spikes->k;
        a.spike_amp = spikes->amp;
    }
    // GM_TRACE_LEVELS=1: device time of every level of both passes on stderr
    static const bool trace = std::getenv("GM_TRACE_LEVELS") != nullptr;
    const int nl = (int)e->levels.size();
    std::vector<cudaEvent_t> ev;
    if (trace) {
        ev.resize(2 * nl + 1);
        for (auto &x : ev) cudaEventCreate(&x);
        cudaEventRecord(ev[0], e->st);
    }
    auto passes = [&](cudaEvent_t *evs) {
        for (int h = 0; h < nl; ++h) {
            launch_solve_forward_level<R>(a, e->levels[h], e->st);
            if (evs) cudaEventRecord(evs[1 + h], e->st);
        }
        cudaEventRecord(e->ev_sm, e->st);
        for (int h = nl - 1; h >= 0; --h) {
            launch_solve_backward_level<R>(a, e->levels[h], e->st);
            if (evs) cudaEventRecord(evs[1 + nl + (nl - 1 - h)], e->st);
        }
    };
    passes(trace ? ev.data() : nullptr);
    if (trace) {
        cudaEventSynchronize(ev[2 * nl]);
        for (int h = 0; h < nl; ++h) {
            float fm = 0, bm = 0;
            cudaEventElapsedTime(&fm, ev[h], ev[1 + h]);
            cudaEventElapsedTime(&bm, ev[nl + (nl - 1 - h)], ev[1 + nl + (nl - 1 - h)]);
            const LevelInfo &L = e->levels[h];
            std::fprintf(stderr, "subst %s level %2d: fronts %5d max_front %4d max_piv %4d max_ring %4d fwd %.3f ms bwd %.3f ms\n",
                         sizeof(R) == 8 ? "c128" : "c64", h, L.count, L.max_front, L.max_piv, L.max_ring, fm, bm);
        }
        for (auto &x : ev) cudaEventDestroy(x);
    }
    cudaEventRecord(e->ev_s1, e->st);
    cudaEventSynchronize(e->ev_s1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev_s0, e->ev_s1);
    e->stats.ms_subst += ms;
    cudaEventElapsedTime(&ms, e->ev_sm, e->ev_s1);
    e->stats.ms_subst_bwd += ms;
    e->stats.n_subst += 1;
}

// Forward-pass pruning mask from a right-hand-side pattern: node v is live
// for right-hand-side group g (32 columns) when a column of the group is
// nonzero on a pivot row of v's subtree -- the owner of every nonzero row
// and that node's ancestors.  Returns the device mask, or NULL (dense).
static const unsigned char *build_mask(gm_engine *e, int nrhs, const RhsPattern *pat) {
    if (!pat || (!pat->per_col && !pat->common) || std::getenv("GM_NO_PRUNE")) return nullptr;
    const Symbolic &sy = e->sym;
    const int nch = (nrhs + 31) / 32, nn = sy.nnodes;
    std::vector<unsigned char> m((size_t)nn * nch, 0);
    auto mark = [&](int row, int g) {
        if (row < 0 || row >= sy.n) return;
        for (int v = sy.owner[row]; v >= 0 && !m[(size_t)v * nch + g]; v = sy.parent[v]) m[(size_t)v * nch + g] = 1;
    };
    if (pat->per_col)
        for (int r = 0; r < std::min(nrhs, pat->ncol); ++r) mark(pat->per_col[r], r / 32);
    for (int i = 0; i < pat->ncommon; ++i)
        for (int g = 0; g < nch; ++g) mark(pat->common[i], g);
    if (e->d_mask.ensure(m.size()) != cudaSuccess) return nullptr;   // fall back to the dense pass
    if (cudaMemcpyAsync(e->d_mask.p, m.data(), m.size(), cudaMemcpyHostToDevice, e->st) != cudaSuccess) return nullptr;
    // the live (front position, slice) pairs of every level, for slices of
    // the width the level's forward pass will use (tuned or default)
    const int tcw_default = solve_slice_width(nrhs, e->cfg.precision == GM_PREC_FP64);
    const bool tuned = !e->lvl_cfg.empty() && e->tuned_nrhs == nrhs;
    std::vector<int2> work;
    e->work_off.assign(e->levels.size() + 1, 0);
    e->work_w.assign(e->levels.size(), tcw_default);
    for (size_t h = 0; h < e->levels.size(); ++h) {
        e->work_off[h] = (int)work.size();
        const int tcw = tuned && e->lvl_cfg[4 * h + 1] ? 8 * e->lvl_cfg[4 * h + 1] : tcw_default;
        e->work_w[h] = tcw;
        const int nslice = (nrhs + tcw - 1) / tcw;
        const LevelInfo &L = e->levels[h];
        for (int t = 0; t < L.count; ++t) {
            const int v = sy.lvl_nodes[L.first + t];
            for (int c = 0; c < nslice; ++c) {
                const int r0 = c * tcw, r1 = std::min(nrhs, r0 + tcw) - 1;
                bool lv = false;
                for (int g = r0 >> 5; g <= (r1 >> 5) && !lv; ++g) lv = m[(size_t)v * nch + g] != 0;
                if (lv) work.push_back(make_int2(t, c));
            }
        }
    }
    e->work_off[e->levels.size()] = (int)work.size();
    e->have_work = e->d_work.ensure((work.size() + 1) * sizeof(int2)) == cudaSuccess &&
                   cudaMemcpyAsync(e->d_work.p, work.data(), work.size() * sizeof(int2), cudaMemcpyHostToDevice,
                                   e->st) == cudaSuccess;
    cudaStreamSynchronize(e->st);   // m and work are released on return
    return e->d_mask.as<unsigned char>();
}

// serialises the GMRES workspace sizing of engines on different host threads
static std::mutex &gmres_alloc_mutex() {
    static std::mutex mu;
    return mu;
}

// GMRES-IR for the matrices `gset` of the batch: restarted GMRES(m) on the
// correction equation M' d = b - M' x, one run per (matrix, right-hand
// side), in FP64 with the working-precision factors as right
// preconditioner (flexible form, gmres.cu).  Each cycle starts from the
// true FP64 residual; a matrix leaves when its worst right-hand side meets
// the target, a cycle ends for a matrix when the least-squares residual
// estimate of each of its right-hand sides is below half the target.  At
// most ir_max_iter iterations per matrix in total.  Updates x in place and
// the matrices' refinement records.
template <class R>
static int gmres_refine(gm_engine *e, int sys, int nrhs, double2 *d_x, const ResidArgs &ra_in,
                        const std::vector<int> &gset) {
    using cd = std::complex<double>;
    const int ng = (int)gset.size();
    if (ng == 0) return GM_OK;
    const int n = e->n;
    const double tol = e->cfg.ir_tol;
    const size_t per = (size_t)n * nrhs;
    const size_t vstride = (size_t)ng * per;   // one Krylov slot holds all ng matrices
    // restart length: the configured one when the Krylov and preconditioned
    // vectors already held fit it; otherwise shortened while they would not
    // fit 80 % of the device memory left, and again while their allocation
    // fails (engines on other host threads allocate at the same time).  The
    // query and the allocation hold a process-wide lock, so concurrent
    // engines see each other's workspaces.
    int m = e->cfg.gmres_restart;
    const auto v_bytes = [&](int mm) { return (size_t)(mm + 1) * vstride * sizeof(double2); };
    const auto z_bytes = [&](int mm) { return (size_t)mm * vstride * sizeof(cplx_any<R>); };
    if (!(e->d_gv.p && e->d_gz.p && e->d_gv.bytes >= v_bytes(m) && e->d_gz.bytes >= z_bytes(m))) {
        std::lock_guard<std::mutex> lock(gmres_alloc_mutex());
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
            const size_t avail = (fr + e->d_gv.bytes + e->d_gz.bytes) / 10 * 8;
            while (m >= 2 && v_bytes(m) + z_bytes(m) > avail) --m;
        }
        for (; m >= 2; --m) {
            if (e->d_gv.ensure(v_bytes(m)) == cudaSuccess && e->d_gz.ensure(z_bytes(m)) == cudaSuccess) break;
            e->d_gv.release();
            e->d_gz.release();
            (void)cudaGetLastError();   // the failed allocation is not an error of this solve
        }
        if (std::getenv("GM_TRACE_REFINEMENT"))
            std::fprintf(stderr, "GMRES workspace: restart %d for %d matrices (%.2f GB free)\n", m, ng, fr / 1e9);
        if (m < 2) return GM_WARNING_NOT_CONVERGED;   // no room: the caller refines with plain sweeps
    }
    const int nblk_r = residual_blocks(e->cfg.nx, e->cfg.ny), nblk_g = (n + 255) / 256;
    const size_t part_words = std::max((size_t)nblk_r * ng * nrhs * 2, (size_t)nblk_g * ng * nrhs * (m + 1) * 2);
    GM_ALLOC(e->d_gpart, part_words * sizeof(double));
    GM_ALLOC(e->d_gnorm, (size_t)ng * nrhs * (m + 1) * 2 * sizeof(double));
    GM_ALLOC(e->d_gcoef, (size_t)ng * nrhs * kGmresStride * sizeof(double2) + (size_t)ng * nrhs * sizeof(double));
    GM_ALLOC(e->d_gmap, 2 * (size_t)ng * sizeof(int));
    double2 *V = e->d_gv.as<double2>();
    cplx_any<R> *Z = e->d_gz.as<cplx_any<R>>();
    double *part = e->d_gpart.as<double>(), *nrm = e->d_gnorm.as<double>();
    double2 *d_coef = e->d_gcoef.as<double2>();
    double *d_scal = reinterpret_cast<double *>(d_coef + (size_t)ng * nrhs * kGmresStride);
    int *d_fm = e->d_gmap.as<int>(), *d_zm = d_fm + ng;

    // per (slot, right-hand side) column: Hessenberg columns, rotations, g
    const int ncol = ng * nrhs;
    std::vector<double> beta((size_t)ncol * (m + 1)), bnorm(ncol);
    std::vector<cd> H((size_t)ncol * (m + 1) * m), cs_sn((size_t)ncol * m * 2), g((size_t)ncol * (m + 1));
    std::vector<char> cdone(ncol);
    std::vector<int> used(ng, 0), kz(ng, 0);
    std::vector<int> live_f, live_z;
    std::vector<double> hn;
    std::vector<double2> hc;
    std::vector<double> hs;
    ResidArgs ra = ra_in;
    ra.xmap = nullptr;

    auto upload_maps = [&](const std::vector<int> &zl) -> int {
        std::vector<int> fz(zl.size());
        for (size_t j = 0; j < zl.size(); ++j) fz[j] = gset[zl[j]];
        GM_CUDA(cudaMemcpy(d_fm, fz.data(), fz.size() * sizeof(int), cudaMemcpyHostToDevice));
        GM_CUDA(cudaMemcpy(d_zm, zl.data(), zl.size() * sizeof(int), cudaMemcpyHostToDevice));
        return GM_OK;
    };
    auto fetch = [&](double *src, size_t words, std::vector<double> &dst) -> int {
        dst.resize(words);
        GM_CUDA(cudaMemcpyAsync(dst.data(), src, words * sizeof(double), cudaMemcpyDeviceToHost, e->st));
        GM_CUDA(cudaStreamSynchronize(e->st));
        return GM_OK;
    };

    std::vector<int> live;   // slots still refined
    for (int z = 0; z < ng; ++z) live.push_back(z);
    for (;;) {
        // true residual V_0 = b - M' x of the live matrices, FP64
        const int nl = (int)live.size();
        int rc;
        if ((rc = upload_maps(live))) return rc;
        ra.fmap = d_fm;
        ra.nfz = nl;
        ra.omap = d_zm;
        ra.r = V;
        const int nb = launch_residual(ra, part, nblk_r, e->st);
        launch_reduce_norms(part, nb, nl * nrhs * 2, nrm, e->st);
        GM_CUDA(cudaGetLastError());
        if ((rc = fetch(nrm, (size_t)nl * nrhs * 2, hn))) return rc;
        std::vector<int> next;
        for (int j = 0; j < nl; ++j) {
            const int z = live[j];
            double wf = 0;
            for (int r = 0; r < nrhs; ++r) {
                const double rr = hn[2 * ((size_t)j * nrhs + r)], bb = hn[2 * ((size_t)j * nrhs + r) + 1];
                if (!std::isfinite(rr)) return fail(GM_ERROR_NONFINITE, "GMRES-IR: non-finite residual");
                const int c = z * nrhs + r;
                beta[(size_t)c * (m + 1)] = std::sqrt(rr);
                bnorm[c] = bb > 0 ? std::sqrt(bb) : 1.0;
                wf = std::max(wf, std::sqrt(rr) / bnorm[c]);
            }
            gm_refine_info &ri = e->refine_info[gset[z]];
            ri.final_residual = wf;
            if (wf > tol && used[z] < e->cfg.ir_max_iter) next.push_back(z);
        }
        if (next.empty()) break;
        if (next.size() != live.size()) {   // V_0 of the remaining slots is in place already
            live.swap(next);
            if ((rc = upload_maps(live))) return rc;
        }
        // one GMRES cycle over the live slots
        for (int z : live) {
            kz[z] = 0;
            for (int r = 0; r < nrhs; ++r) {
                const int c = z * nrhs + r;
                const double b0 = beta[(size_t)c * (m + 1)];
                cdone[c] = !(b0 > 0.5 * tol * bnorm[c]);
                std::fill(g.begin() + (size_t)c * (m + 1), g.begin() + (size_t)(c + 1) * (m + 1), cd(0));
                std::fill(H.begin() + (size_t)c * (m + 1) * m, H.begin() + (size_t)(c + 1) * (m + 1) * m, cd(0));
                g[(size_t)c * (m + 1)] = b0;
            }
        }
        std::vector<int> inner = live;
        const int max_j = std::min(m, e->cfg.ir_max_iter);
        for (int jj = 0; jj < max_j && !inner.empty(); ++jj) {
            const int ni = (int)inner.size();
            if ((rc = upload_maps(inner))) return rc;
            // Z_jj = (R)(V_jj / beta_jj)
            hs.assign((size_t)ni * nrhs, 0.0);
            for (int j = 0; j < ni; ++j)
                for (int r = 0; r < nrhs; ++r) {
                    const int c = inner[j] * nrhs + r;
                    const double b = beta[(size_t)c * (m + 1) + jj];
                    hs[(size_t)j * nrhs + r] = (!cdone[c] && b > 0) ? 1.0 / b : 0.0;
                }
            GM_CUDA(cudaMemcpy(d_scal, hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice));
            launch_scale_down<R>(V + jj * vstride, Z + jj * vstride, d_scal, d_zm, ni, n, nrhs, e->st);
            // Z_jj <- M~^-1 Z_jj (working-precision substitution in place)
            substitute<R>(e, Z + jj * vstride, nrhs, sys, nullptr, d_fm, ni, d_zm);
            // V_jj+1 = M' Z_jj (FP64)
            ResidArgs pa = ra;
            pa.fmap = d_fm; pa.nfz = ni; pa.xmap = d_zm; pa.omap = d_zm;
            launch_matvec<R>(pa, Z + jj * vstride, V + (jj + 1) * vstride, part, nblk_r, e->st);
            // h_i = <v_i, w>: dots with the unnormalised V_i
            const int nv = jj + 1;
            const int nbd = launch_dots(V, vstride, nv, V + (jj + 1) * vstride, d_zm, ni, n, nrhs, part, e->st);
            launch_reduce_norms(part, nbd, ni * nrhs * (nv + 1) * 2, nrm, e->st);
            GM_CUDA(cudaGetLastError());
            if ((rc = fetch(nrm, (size_t)ni * nrhs * (nv + 1) * 2, hn))) return rc;
            hc.assign((size_t)ni * nrhs * kGmresStride, make_double2(0.0, 0.0));
            for (int j = 0; j < ni; ++j)
                for (int r = 0; r < nrhs; ++r) {
                    const int c = inner[j] * nrhs + r;
                    if (cdone[c]) continue;   // its coefficients stay 0: W is left as it is
                    for (int i = 0; i < nv; ++i) {
                        const double *p = &hn[(((size_t)j * nrhs + r) * (nv + 1) + i) * 2];
                        const double bi = beta[(size_t)c * (m + 1) + i];
                        const cd h = cd(p[0], p[1]) / bi;   // <V_i / beta_i, w>
                        H[((size_t)c * (m + 1) + i) * m + jj] = h;
                        const cd co = h / bi;
                        hc[((size_t)j * nrhs + r) * kGmresStride + i] = make_double2(co.real(), co.imag());
                    }
                }
            GM_CUDA(cudaMemcpy(d_coef, hc.data(), hc.size() * sizeof(double2), cudaMemcpyHostToDevice));
            const int nbu = launch_gs_update(V, vstride, nv, V + (jj + 1) * vstride, d_coef, d_zm, ni, n, nrhs, part,
                                             e->st);
            launch_reduce_norms(part, nbu, ni * nrhs, nrm, e->st);
            GM_CUDA(cudaGetLastError());
            if ((rc = fetch(nrm, (size_t)ni * nrhs, hn))) return rc;
            // Givens rotations of column jj and the residual estimates
            std::vector<int> still;
            for (int j = 0; j < ni; ++j) {
                const int z = inner[j];
                bool all_done = true;
                for (int r = 0; r < nrhs; ++r) {
                    const int c = z * nrhs + r;
                    if (cdone[c]) continue;
                    const double hnext = std::sqrt(std::max(hn[(size_t)j * nrhs + r], 0.0));
                    beta[(size_t)c * (m + 1) + jj + 1] = hnext;
                    cd *Hc = &H[(size_t)c * (m + 1) * m];
                    cd *rot = &cs_sn[(size_t)c * m * 2];
                    for (int i = 0; i < jj; ++i) {   // earlier rotations
                        const cd cs = rot[2 * i], sn = rot[2 * i + 1];
                        const cd a = Hc[i * m + jj], b = Hc[(i + 1) * m + jj];
                        Hc[i * m + jj] = cs * a + sn * b;
                        Hc[(i + 1) * m + jj] = -std::conj(sn) * a + cs * b;
                    }
                    const cd a = Hc[jj * m + jj];
                    const double t = std::hypot(std::abs(a), hnext);
                    cd cs, sn;
                    if (std::abs(a) == 0.0) {
                        cs = 0.0;
                        sn = 1.0;
                    } else {
                        cs = std::abs(a) / t;
                        sn = (a / std::abs(a)) * hnext / t;
                    }
                    rot[2 * jj] = cs;
                    rot[2 * jj + 1] = sn;
                    Hc[jj * m + jj] = cs * a + sn * hnext;
                    Hc[(jj + 1) * m + jj] = 0.0;
                    cd *gc = &g[(size_t)c * (m + 1)];
                    gc[jj + 1] = -std::conj(sn) * gc[jj];
                    gc[jj] = cs * gc[jj];
                    if (std::abs(gc[jj + 1]) <= 0.5 * tol * bnorm[c] || !(hnext > 0)) cdone[c] = 1;
                    else all_done = false;
                }
                kz[z] = jj + 1;
                if (!all_done) still.push_back(z);
            }
            if (std::getenv("GM_TRACE_REFINEMENT")) {
                std::fprintf(stderr, "GMRES iteration %d: largest estimated relative residual per matrix", jj + 1);
                for (int j = 0; j < ni; ++j) {
                    double w = 0;
                    for (int r = 0; r < nrhs; ++r) {
                        const int c = inner[j] * nrhs + r;
                        w = std::max(w, std::abs(g[(size_t)c * (m + 1) + jj + 1]) / bnorm[c]);
                    }
                    std::fprintf(stderr, " [%d] %.2e", gset[inner[j]], w);
                }
                std::fprintf(stderr, "\n");
            }
            inner.swap(still);
        }
        // x += sum_i y_i Z_i with R y = g (upper triangular), per matrix
        for (int z : live) {
            const int k = kz[z];
            if (k == 0) continue;
            hc.assign((size_t)nrhs * kGmresStride, make_double2(0.0, 0.0));
            for (int r = 0; r < nrhs; ++r) {
                const int c = z * nrhs + r;
                const cd *Hc = &H[(size_t)c * (m + 1) * m];
                const cd *gc = &g[(size_t)c * (m + 1)];
                // columns that met the estimate early have k_c < k entries;
                // their trailing rows are 0, so solve over the nonzero part
                int kc = k;
                while (kc > 0 && Hc[(kc - 1) * m + (kc - 1)] == cd(0)) --kc;
                std::vector<cd> y(kc);
                for (int i = kc - 1; i >= 0; --i) {
                    cd acc = gc[i];
                    for (int q = i + 1; q < kc; ++q) acc -= Hc[i * m + q] * y[q];
                    y[i] = acc / Hc[i * m + i];
                }
                for (int i = 0; i < kc; ++i)
                    hc[(size_t)r * kGmresStride + i] = make_double2(y[i].real(), y[i].imag());
            }
            GM_CUDA(cudaMemcpy(d_coef, hc.data(), hc.size() * sizeof(double2), cudaMemcpyHostToDevice));
            const int fz = gset[z];
            GM_CUDA(cudaMemcpy(d_fm, &fz, sizeof(int), cudaMemcpyHostToDevice));
            GM_CUDA(cudaMemcpy(d_zm, &z, sizeof(int), cudaMemcpyHostToDevice));
            launch_x_update<R>(d_x, Z, vstride, k, d_coef, d_fm, d_zm, 1, n, nrhs, e->st);
            GM_CUDA(cudaGetLastError());
            used[z] += k;
            gm_refine_info &ri = e->refine_info[fz];
            ri.sweeps += k;
            ri.method = GM_REFINE_GMRES;
            GM_CUDA(cudaStreamSynchronize(e->st));   // d_coef / maps are rewritten next
        }
    }
    return GM_OK;
}

// x (device, [nf][n][nrhs] c128) = M'^{-1} b with FP64 refinement; b, x device.
// The first substitution prunes the forward pass by `pattern` when given;
// the refinement sweeps (dense residuals) do not.
int engine_solve_device(gm_engine *e, int sys, int nrhs, double2 *d_x, const double2 *d_b, const RhsPattern *pattern,
                        const SpikeRhs *spikes) {
    if (!d_b && !(spikes && spikes->k && spikes->amp)) return fail(GM_ERROR_INVALID, "solve: no right-hand side");
    const size_t cnt = (size_t)e->nf * e->n * nrhs;
    const bool fp64 = e->cfg.precision == GM_PREC_FP64;
    GM_ALLOC(e->d_t, cnt * e->csize());
    GM_ALLOC(e->d_w, (size_t)e->nf * e->sym.rhs_total * nrhs * e->csize());
    const int nblk_max = residual_blocks(e->cfg.nx, e->cfg.ny);
    GM_ALLOC(e->d_part, (size_t)nblk_max * e->nf * nrhs * 2 * sizeof(double));
    GM_ALLOC(e->d_norm, (size_t)e->nf * nrhs * 2 * sizeof(double));

    cudaEvent_t t0 = e->ev0, t1 = e->ev1;
    e->stats.ms_subst = 0;
    e->stats.ms_subst_bwd = 0;
    e->stats.n_subst = 0;
    GM_CUDA(cudaEventRecord(t0, e->st));
    // initial solve in working precision: in FP64 in place in x (b copied
    // into it), in complex64 in the work buffer and then added into x = 0
    const unsigned char *mask = build_mask(e, nrhs, pattern);
    const bool implicit = !d_b;
    // FP64 with implicit spikes and a pruning mask: x is not cleared, the
    // passes take b from the spike list (pruned fronts: y = 0)
    const bool lazy_b = implicit && fp64 && mask;
    if (implicit && !lazy_b) launch_spikes(d_x, e->n, e->nf, nrhs, spikes->k, spikes->amp, e->st);   // x = b
    if (fp64) {
        if (!implicit) GM_CUDA(cudaMemcpyAsync(d_x, d_b, cnt * sizeof(double2), cudaMemcpyDeviceToDevice, e->st));
        substitute<double>(e, d_x, nrhs, sys, mask, nullptr, 0, nullptr, lazy_b ? spikes : nullptr);
    } else {
        launch_convert_down<float>(implicit ? d_x : d_b, e->d_t.p, cnt, e->st);
        GM_CUDA(cudaMemsetAsync(d_x, 0, cnt * sizeof(double2), e->st));
        substitute<float>(e, e->d_t.p, nrhs, sys, mask);
        launch_add_up<float>(d_x, e->d_t.p, cnt, e->st);
    }
    GM_CUDA(cudaGetLastError());
    GM_CUDA(cudaEventRecord(t1, e->st));
    GM_CUDA(cudaEventSynchronize(t1));
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    e->stats.ms_solve = ms;

    // Refinement, per matrix: r = b - M' x (FP64), x += M'^{-1} r (working
    // precision), until the matrix's worst right-hand side meets the target.
    // A matrix that has met it leaves the sweeps: the residual, substitution
    // and update kernels of the next sweep run over the remaining matrices
    // only (their list is the launch's fmap).
    ResidArgs ra{};
    ra.nx = e->cfg.nx; ra.ny = e->cfg.ny; ra.n = e->n; ra.nf = e->nf; ra.nrhs = nrhs; ra.ldr = nrhs;
    ra.A = e->d_A.as<double2>(); ra.x = d_x; ra.b = d_b; ra.r = nullptr;
    ra.op_mode = e->cfg.op_mode; ra.trans = sys;
    if (implicit) {
        ra.spike_k = spikes->k;
        ra.spike_amp = spikes->amp;
    }
    GM_ALLOC(e->d_fmap, 2 * (size_t)e->nf * sizeof(int));
    int *d_act = e->d_fmap.as<int>();
    std::vector<int> &act = e->h_fmap;
    act.resize(e->nf);
    for (int f = 0; f < e->nf; ++f) act[f] = f;
    std::vector<double> norms((size_t)e->nf * nrhs * 2);
    std::vector<double> prev_res(e->nf, 0.0);
    e->refine_info.assign(e->nf, gm_refine_info{0.0, 0.0, 0, GM_REFINE_NONE});
    double worst = 0;
    int it = 0;
    GM_CUDA(cudaEventRecord(t0, e->st));
    for (;; ++it) {
        const int na = (int)act.size();
        GM_CUDA(cudaMemcpyAsync(d_act, act.data(), na * sizeof(int), cudaMemcpyHostToDevice, e->st));
        ra.fmap = d_act;
        ra.nfz = na;
        ra.omap = nullptr;
        ra.xmap = nullptr;
        // residual straight into the working-precision right-hand side; the
        // first check of FP64 factors normally passes, so it computes the
        // norms only and the residual is formed again if a sweep follows
        void *rhs = (fp64 && it == 0) ? nullptr : e->d_t.p;
        const int nblk = fp64 ? launch_residual_t<double>(ra, rhs, e->d_part.as<double>(), nblk_max, e->st)
                              : launch_residual_t<float>(ra, rhs, e->d_part.as<double>(), nblk_max, e->st);
        const int cntn = na * nrhs * 2;
        launch_reduce_norms(e->d_part.as<double>(), nblk, cntn, e->d_norm.as<double>(), e->st);
        GM_CUDA(cudaGetLastError());
        GM_CUDA(cudaMemcpyAsync(norms.data(), e->d_norm.p, cntn * sizeof(double), cudaMemcpyDeviceToHost, e->st));
        GM_CUDA(cudaStreamSynchronize(e->st));
        bool finite = true;
        std::vector<int> next;
        for (int z = 0; z < na; ++z) {
            const int f = act[z];
            double wf = 0;
            for (int r = 0; r < nrhs; ++r) {
                const double rr = norms[2 * ((size_t)z * nrhs + r)], bb = norms[2 * ((size_t)z * nrhs + r) + 1];
                if (!std::isfinite(rr)) finite = false;
                wf = std::max(wf, bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr));
            }
            gm_refine_info &ri = e->refine_info[f];
            if (it == 0) ri.first_residual = wf;
            ri.final_residual = wf;
            if (wf > e->cfg.ir_tol) next.push_back(f);
        }
        if (!finite) {
            e->stats.ir_iterations = it;
            e->stats.ir_residual = NAN;
            return fail(GM_ERROR_NONFINITE, "non-finite residual after %d refinement sweeps", it);
        }
        worst = 0;
        for (const gm_refine_info &ri : e->refine_info) worst = std::max(worst, ri.final_residual);
        if (std::getenv("GM_TRACE_REFINEMENT")) {
            std::fprintf(stderr, "refinement sweep %d: max relative residual %.3e; per matrix", it, worst);
            for (const gm_refine_info &ri : e->refine_info) std::fprintf(stderr, " %.1e", ri.final_residual);
            std::fprintf(stderr, "\n");
        }
        if (next.empty() || it >= e->cfg.ir_max_iter) break;
        // Matrices that go on with GMRES-IR: all of them in GMRES mode; in
        // auto mode those whose plain sweeps cannot reach the target within
        // the sweeps left at the contraction of the last one (or did not
        // contract at all).  The first check has no contraction yet, so
        // every matrix starts with a plain sweep; plain sweeps need no
        // Krylov vectors, which matters when many engines share the device.
        std::vector<int> gset, irset;
        for (int f : next) {
            const gm_refine_info &ri = e->refine_info[f];
            bool to_gmres = e->cfg.refine == GM_REFINE_MODE_GMRES;
            if (e->cfg.refine == GM_REFINE_MODE_AUTO && it > 0 && !fp64) {   // FP64 factors: plain sweeps
                const double rho = prev_res[f] > 0 ? ri.final_residual / prev_res[f] : 1.0;
                const double need = std::log(e->cfg.ir_tol / ri.final_residual);
                to_gmres = !(rho < 1.0) || need / std::log(rho) > (double)(e->cfg.ir_max_iter - it);
            }
            (to_gmres ? gset : irset).push_back(f);
        }
        for (int f : next) prev_res[f] = e->refine_info[f].final_residual;
        if (!gset.empty()) {
            const int grc = fp64 ? gmres_refine<double>(e, sys, nrhs, d_x, ra, gset)
                                 : gmres_refine<float>(e, sys, nrhs, d_x, ra, gset);
            if (grc == GM_WARNING_NOT_CONVERGED) {   // no room for the Krylov vectors: plain sweeps
                irset.insert(irset.end(), gset.begin(), gset.end());
                std::sort(irset.begin(), irset.end());
                gset.clear();
            } else if (grc) {
                e->stats.ir_iterations = it;
                e->stats.ir_residual = NAN;
                return grc;
            }
        }
        if (irset.empty()) {
            worst = 0;
            for (const gm_refine_info &ri : e->refine_info) worst = std::max(worst, ri.final_residual);
            ++it;
            break;
        }
        // the remaining matrices: their residual is in t (formed again for
        // the FP64 path, whose first check formed norms only)
        const int nn = (int)irset.size();
        act.swap(irset);
        ra.omap = nullptr;
        ra.xmap = nullptr;
        ra.r = nullptr;
        GM_CUDA(cudaMemcpyAsync(d_act, act.data(), nn * sizeof(int), cudaMemcpyHostToDevice, e->st));
        ra.nfz = nn;
        if (!rhs) launch_residual_t<double>(ra, e->d_t.p, e->d_part.as<double>(), nblk_max, e->st);
        const size_t per_f = (size_t)e->n * nrhs;
        if (fp64) {
            substitute<double>(e, e->d_t.p, nrhs, sys, nullptr, d_act, nn);
            launch_add_up_f<double>(d_x, e->d_t.p, per_f, d_act, nn, e->st);
        } else {
            substitute<float>(e, e->d_t.p, nrhs, sys, nullptr, d_act, nn);
            launch_add_up_f<float>(d_x, e->d_t.p, per_f, d_act, nn, e->st);
        }
        for (int f : act) {
            e->refine_info[f].sweeps += 1;
            e->refine_info[f].method = GM_REFINE_IR;
        }
    }
    GM_CUDA(cudaEventRecord(t1, e->st));
    GM_CUDA(cudaEventSynchronize(t1));
    cudaEventElapsedTime(&ms, t0, t1);
    e->stats.ms_refine = ms;
    e->stats.ir_iterations = it;
    e->stats.ir_residual = worst;
    return worst <= e->cfg.ir_tol ? GM_OK : GM_WARNING_NOT_CONVERGED;
}

}  // namespace gm

namespace gm {

// Device time of every level of one forward and one backward pass over
// right-hand sides held in xT (all dense), with the engine's current
// per-level tile table.
template <class R>
static void time_levels(gm_engine *e, void *xT, int nrhs, std::vector<float> &fwd, std::vector<float> &bwd) {
    const int nl = (int)e->levels.size();
    SolveArgs<R> a{};
    a.s = e->dsym;
    a.front = e->d_front.p;
    a.pivsrc = e->cfg.pivot_tol > 0 ? e->d_pivsrc.as<unsigned char>() : nullptr;
    a.x = xT;
    a.w = e->d_w.p;
    a.nf = e->nf;
    a.nrhs = nrhs;
    a.ldr = nrhs;
    const int nchunk = (nrhs + 31) / 32;
    a.rch = (nrhs + nchunk - 1) / nchunk;
    a.lvl_cfg = e->lvl_cfg.data();
    std::vector<cudaEvent_t> ev(2 * nl + 1);
    for (auto &x : ev) cudaEventCreate(&x);
    cudaEventRecord(ev[0], e->st);
    for (int h = 0; h < nl; ++h) {
        launch_solve_forward_level<R>(a, e->levels[h], e->st);
        cudaEventRecord(ev[1 + h], e->st);
    }
    for (int h = nl - 1; h >= 0; --h) {
        launch_solve_backward_level<R>(a, e->levels[h], e->st);
        cudaEventRecord(ev[1 + nl + (nl - 1 - h)], e->st);
    }
    cudaEventSynchronize(ev[2 * nl]);
    fwd.assign(nl, 0.f);
    bwd.assign(nl, 0.f);
    for (int h = 0; h < nl; ++h) {
        cudaEventElapsedTime(&fwd[h], ev[h], ev[1 + h]);
        cudaEventElapsedTime(&bwd[h], ev[nl + (nl - 1 - h)], ev[1 + nl + (nl - 1 - h)]);
    }
    for (auto &x : ev) cudaEventDestroy(x);
}

}  // namespace gm

extern "C" int gm_autotune(gm_engine *e, int nrhs, int reps) {
    if (!e || nrhs <= 0) return fail(GM_ERROR_INVALID, "gm_autotune: bad argument");
    if (!e->factored) return fail(GM_ERROR_STATE, "gm_autotune: no factorisation (gm_factor)");
    GM_CUDA(cudaSetDevice(e->device));
    if (reps <= 0) reps = 2;
    const bool fp64 = e->cfg.precision == GM_PREC_FP64;
    const size_t cnt = (size_t)e->nf * e->n * nrhs;
    GM_ALLOC(e->d_t, cnt * e->csize());
    GM_ALLOC(e->d_w, (size_t)e->nf * e->sym.rhs_total * nrhs * e->csize());
    GM_CUDA(cudaMemsetAsync(e->d_t.p, 0, cnt * e->csize(), e->st));   // the pass's cost does not depend on the values
    const int nl = (int)e->levels.size();
    // per level, each pass direction: the fastest of the candidate tiles
    // (row height 32 / 64 x slice width 32 / 40 columns), best of reps
    // timings; a candidate replaces the built-in choice (lvl_cfg 0) only
    // when it is at least 3 % faster, so timing noise keeps the default
    const int cand[5][2] = {{0, 0}, {32, 4}, {64, 4}, {32, 5}, {64, 5}};
    std::vector<float> best_f(nl, 1e30f), best_b(nl, 1e30f);
    std::vector<int> pick(4 * nl, 0);
    std::vector<float> tf, tb;
    auto time_pass = [&](std::vector<float> &sf, std::vector<float> &sb) {
        sf.assign(nl, 1e30f);
        sb.assign(nl, 1e30f);
        for (int r = 0; r < reps; ++r) {   // best of reps (the first run also loads the kernels)
            if (fp64) gm::time_levels<double>(e, e->d_t.p, nrhs, tf, tb);
            else gm::time_levels<float>(e, e->d_t.p, nrhs, tf, tb);
            for (int h = 0; h < nl; ++h) { sf[h] = std::min(sf[h], tf[h]); sb[h] = std::min(sb[h], tb[h]); }
        }
    };
    for (const auto &c : cand) {
        e->lvl_cfg.assign(4 * nl, 0);
        for (int h = 0; h < nl; ++h) {
            e->lvl_cfg[4 * h + 0] = c[0]; e->lvl_cfg[4 * h + 1] = c[1];
            e->lvl_cfg[4 * h + 2] = c[0]; e->lvl_cfg[4 * h + 3] = c[1];
        }
        std::vector<float> sf, sb;
        time_pass(sf, sb);
        const float margin = c[0] ? 0.97f : 1.0f;
        for (int h = 0; h < nl; ++h) {
            // forward levels of fronts with at most 32 pivots keep 32-row
            // tiles: only that kernel runs the pruned first pass of
            // spike right-hand sides from a work list
            const bool fwd_ok = !(c[0] == 64 && e->levels[h].max_piv <= 32);
            if (fwd_ok && sf[h] < margin * best_f[h]) {
                best_f[h] = sf[h]; pick[4 * h + 0] = c[0]; pick[4 * h + 1] = c[1];
            }
            if (sb[h] < margin * best_b[h]) { best_b[h] = sb[h]; pick[4 * h + 2] = c[0]; pick[4 * h + 3] = c[1]; }
        }
    }
    // the per-level picks must also win over whole passes (a level's tiles
    // change what the next level finds in L2): interleaved timings of the
    // picked table against the built-in choice, the faster total kept
    {
        std::vector<float> sf, sb;
        float t_pick = 1e30f, t_def = 1e30f;
        for (int r = 0; r < 2; ++r) {
            e->lvl_cfg = pick;
            time_pass(sf, sb);
            float t = 0;
            for (int h = 0; h < nl; ++h) t += sf[h] + sb[h];
            t_pick = std::min(t_pick, t);
            e->lvl_cfg.assign(4 * nl, 0);
            time_pass(sf, sb);
            t = 0;
            for (int h = 0; h < nl; ++h) t += sf[h] + sb[h];
            t_def = std::min(t_def, t);
        }
        if (!(t_pick < t_def)) pick.assign(4 * nl, 0);
    }
    // the table names every level's tiles: built-in choices resolved
    const int b_def = gm::solve_slice_width(nrhs, fp64) / 8;
    for (int h = 0; h < nl; ++h)
        for (int d = 0; d < 2; ++d)
            if (pick[4 * h + 2 * d] == 0) {
                pick[4 * h + 2 * d] = gm::solve_level_rt(e->levels[h]);
                pick[4 * h + 2 * d + 1] = b_def;
            }
    GM_CUDA(cudaGetLastError());
    e->lvl_cfg = pick;
    e->tuned_nrhs = nrhs;
    if (std::getenv("GM_TRACE_LEVELS"))
        for (int h = 0; h < nl; ++h)
            std::fprintf(stderr, "autotune level %2d: forward rt %d slice %d (%.3f ms), backward rt %d slice %d (%.3f ms)\n",
                         h, pick[4 * h], 8 * pick[4 * h + 1], best_f[h], pick[4 * h + 2], 8 * pick[4 * h + 3], best_b[h]);
    return GM_OK;
}

extern "C" int gm_autotune_table(const gm_engine *e, int *nrhs, int *table, int nlevels) {
    if (!e || !nrhs) return fail(GM_ERROR_INVALID, "gm_autotune_table: bad argument");
    *nrhs = e->tuned_nrhs;
    if (table && nlevels > 0)
        for (int i = 0; i < 4 * std::min(nlevels, (int)e->levels.size()); ++i)
            table[i] = i < (int)e->lvl_cfg.size() ? e->lvl_cfg[i] : 0;
    return GM_OK;
}

extern "C" int gm_set_refine(gm_engine *e, int refine, int gmres_restart) {
    if (!e) return fail(GM_ERROR_INVALID, "gm_set_refine: null engine");
    if (refine < GM_REFINE_MODE_AUTO || refine > GM_REFINE_MODE_GMRES)
        return fail(GM_ERROR_INVALID, "unknown refinement mode %d", refine);
    if (gmres_restart < 0) return fail(GM_ERROR_INVALID, "GMRES restart length must be >= 0");
    e->cfg.refine = refine;
    e->cfg.gmres_restart = gmres_restart == 0 || gmres_restart > gm::kGmresMaxRestart ? gm::kGmresMaxRestart
                                                                                        : gmres_restart;
    return GM_OK;
}

extern "C" int gm_refine_report(const gm_engine *e, int nmat, gm_refine_info *out) {
    if (!e || !out) return fail(GM_ERROR_INVALID, "gm_refine_report: null argument");
    if (nmat != (int)e->refine_info.size())
        return fail(GM_ERROR_INVALID, "gm_refine_report: the last solve covered %d matrices, not %d",
                    (int)e->refine_info.size(), nmat);
    for (int f = 0; f < nmat; ++f) out[f] = e->refine_info[f];
    return GM_OK;
}

extern "C" int gm_solve(gm_engine *e, int sys, int nrhs, const double *b, double *x) {
    if (!e || !b || !x || nrhs <= 0) return fail(GM_ERROR_INVALID, "gm_solve: bad argument");
    if (sys != GM_SYS_A && sys != GM_SYS_AT) return fail(GM_ERROR_INVALID, "gm_solve: unknown sys %d", sys);
    if (!e->factored) return fail(GM_ERROR_STATE, "gm_solve: no factorisation (gm_factor)");
    GM_CUDA(cudaSetDevice(e->device));
    const size_t cnt = (size_t)e->nf * e->n * nrhs;
    GM_ALLOC(e->d_b, cnt * sizeof(double2));
    GM_ALLOC(e->d_x, cnt * sizeof(double2));
    GM_CUDA(cudaMemcpyAsync(e->d_b.p, b, cnt * sizeof(double2), cudaMemcpyDefault, e->st));
    int rc = gm::engine_solve_device(e, sys, nrhs, e->d_x.as<double2>(), e->d_b.as<double2>());
    if (rc < 0) return rc;
    GM_CUDA(cudaMemcpyAsync(x, e->d_x.p, cnt * sizeof(double2), cudaMemcpyDefault, e->st));
    GM_CUDA(cudaStreamSynchronize(e->st));
    return rc;
}
