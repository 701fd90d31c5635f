// gm_forward / gm_grad_obj / gm_obj: the per-frequency drivers of the
// reference (forward_shot_AC, grad_obj_AC, obj_AC and their TE/SH twins)
// over every shot and every frequency of the factorised batch at once.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.hpp"
#include "host_setup.h"
#include "kernels_epi.cuh"

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

// iround of fd.h:20 applied to a float quotient, as sources()/receiver() do
int iround_div(float x, float dh) {
    const float q = x / dh;
    return (int)std::floor((double)q + 0.5);
}

struct Geometry {
    std::vector<int> ksrc;   // RHS index of each shot (RHS_source_AC.c:32)
    std::vector<int> krec;   // grid index read for each receiver before the vec2mat shift
    std::vector<int> kadj;   // RHS index of each adjoint source (RHS_source_AC_adj.c:28)
};

int make_geometry(const gm_engine *e, int ns, const float *sx, const float *sy, int ntr, const int32_t *rx,
                  const int32_t *ry, Geometry &g) {
    const gm_config &c = e->cfg;
    const int n = e->n;
    g.ksrc.resize(ns);
    for (int s = 0; s < ns; ++s) {
        const int nxs = iround_div(sx[s], c.dh) + c.npml;
        const int nys = iround_div(sy[s], c.dh) + e->fsshift;
        const long k = (long)nxs + (long)(nys - 1) * c.nx;
        if (k < 0 || k >= n)
            return fail(GM_ERROR_INVALID, "shot %d at (%g, %g) m falls outside the %d x %d grid", s, sx[s], sy[s], c.nx, c.ny);
        g.ksrc[s] = (int)k;
    }
    g.krec.resize(ntr);
    g.kadj.resize(ntr);
    for (int t = 0; t < ntr; ++t) {
        const long kr = (long)(ry[t] + e->fsshift - 1) * c.nx + (rx[t] + c.npml - 1);
        const long ka = (long)(rx[t] + c.npml) + (long)(ry[t] + e->fsshift - 1) * c.nx;
        if (kr < 0 || kr >= n || ka < 0 || ka >= n)
            return fail(GM_ERROR_INVALID, "receiver %d at grid (%d, %d) falls outside the grid", t, rx[t], ry[t]);
        g.krec[t] = (int)kr;
        g.kadj[t] = (int)ka;
    }
    return GM_OK;
}

template <class T>
int upload(gm::DevBuf &buf, const std::vector<T> &v, cudaStream_t st) {
    GM_ALLOC(buf, v.size() * sizeof(T) + 16);
    if (!v.empty()) GM_CUDA(cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return GM_OK;
}

// spike right-hand sides of every shot and frequency into e->d_b, forward solve into xout;
// the spike amplitude is that of src_physics's source routine (RHS_source_AC / _TE)
int forward_solve(gm_engine *e, int ns, const Geometry &g, double2 *xout, int src_physics = 0) {
    const int nf = e->nf, n = e->n;
    if (!src_physics) src_physics = e->cfg.physics;
    std::vector<double2> amp(nf);
    if (!e->wavelet.empty() && e->wavelet.size() != 2 * (size_t)nf)
        return fail(GM_ERROR_STATE, "the source wavelet holds %d amplitudes, the batch %d matrices",
                    (int)(e->wavelet.size() / 2), nf);
    for (int f = 0; f < nf; ++f) {
        double a[2];
        if (e->wavelet.empty()) gmh_source_amp(src_physics, e->freqs[f], e->cfg.s, e->cfg.dh, a);
        else gmh_wavelet_amp(&e->wavelet[2 * (size_t)f], e->cfg.dh, a);
        amp[f] = make_double2(a[0], a[1]);
    }
    int rc;
    if ((rc = upload(e->d_src_k, g.ksrc, e->st))) return rc;
    gm::DevBuf amp_buf;
    if ((rc = upload(amp_buf, amp, e->st))) return rc;
    (void)n;
    gm::RhsPattern pat;   // one spike per shot: prune the forward pass
    pat.per_col = g.ksrc.data();
    pat.ncol = ns;
    gm::SpikeRhs sp;      // and never form the dense right-hand sides
    sp.k = e->d_src_k.as<int>();
    sp.amp = amp_buf.as<double2>();
    rc = gm::engine_solve_device(e, GM_SYS_A, ns, xout, nullptr, &pat, &sp);
    GM_CUDA(cudaStreamSynchronize(e->st));  // amp_buf is released on return
    return rc;
}

// cp_grad_frame's taper (coefficient and number of passes per grid point) on the device
int ensure_frame(gm_engine *e) {
    if (e->d_frame.p) return GM_OK;
    const int n = e->n;
    std::vector<float> coef(n);
    std::vector<unsigned char> passes(n);
    gmh_grad_frame(e->cfg.nx, e->cfg.ny, e->cfg.npml, e->cfg.free_surf, coef.data(), passes.data());
    int rc;
    if ((rc = upload(e->d_frame, coef, e->st))) return rc;
    if ((rc = upload(e->d_frame_pass, passes, e->st))) return rc;
    GM_CUDA(cudaStreamSynchronize(e->st));   // the host vectors are released on return
    return GM_OK;
}

int single_model(const gm_engine *e, const char *who) {
    for (int m : e->models)
        if (m != e->models[0])
            return fail(GM_ERROR_STATE, "%s: the factorised matrices come from different models", who);
    return GM_OK;
}

int check_ready(const gm_engine *e, int ns, int ntr) {
    if (!e) return fail(GM_ERROR_INVALID, "null engine");
    if (!e->factored) return fail(GM_ERROR_STATE, "no factorisation (call gm_factor first)");
    if (e->values_only)
        return fail(GM_ERROR_STATE, "the factors come from gm_factor_values: no frequencies or model to model shots with");
    if (ns <= 0 || ntr < 0) return fail(GM_ERROR_INVALID, "need at least one shot (nshots=%d, ntr=%d)", ns, ntr);
    return GM_OK;
}

// forward + seismograms (cal kept in e->d_res as complex128) ; returns solve status
int forward_and_seis(gm_engine *e, int ns, const Geometry &g, int ntr, float *seis_out) {
    const int nf = e->nf, n = e->n;
    GM_ALLOC(e->d_xf, (size_t)nf * n * ns * sizeof(double2));
    e->xf_ns = 0;
    e->xa_ns = 0;
    const int rc = forward_solve(e, ns, g, e->d_xf.as<double2>());
    if (rc < 0) return rc;
    e->xf_ns = ns;
    if (ntr > 0) {
        int rc2;
        if ((rc2 = upload(e->d_rec_k, g.krec, e->st))) return rc2;
        const size_t cnt = (size_t)nf * ns * ntr;
        GM_ALLOC(e->d_res, 2 * cnt * sizeof(double2));   // cal | res
        GM_ALLOC(e->d_seis, cnt * sizeof(float2));
        gm::launch_gather_seis(e->d_xf.as<double2>(), n, nf, ns, ntr, e->d_rec_k.as<int>(), e->d_seis.as<float2>(),
                               e->d_res.as<double2>(), e->st);
        GM_CUDA(cudaGetLastError());
        if (seis_out) GM_CUDA(cudaMemcpyAsync(seis_out, e->d_seis.p, cnt * sizeof(float2), cudaMemcpyDefault, e->st));
    }
    return rc;
}

// residuals and misfit; leaves res in the second half of e->d_res and the
// source estimates w/|w| on the host
int residuals(gm_engine *e, int ns, int ntr, const float *pobs, int stf_inv, int misfit, double &l2,
              std::vector<double2> &stfu, std::vector<double> *l2_each = nullptr) {
    const int nf = e->nf;
    const size_t cnt = (size_t)nf * ns * ntr;
    const int nfs = nf * ns;
    GM_ALLOC(e->d_misc, cnt * sizeof(float2) + (size_t)nfs * (sizeof(double) + sizeof(double2)) + 64);
    float2 *obs = e->d_misc.as<float2>();
    double *l2p = reinterpret_cast<double *>(obs + cnt);
    double2 *stf = reinterpret_cast<double2 *>(l2p + nfs + (nfs & 1));
    GM_CUDA(cudaMemcpyAsync(obs, pobs, cnt * sizeof(float2), cudaMemcpyDefault, e->st));
    double2 *cal = e->d_res.as<double2>(), *res = cal + cnt;
    // GM_OP_EXACT forms the exact residual: no zeroing of tiny observed samples
    const int zeroing = e->cfg.op_mode == GM_OP_EXACT ? 0 : 1;
    gm::launch_residual_shot(cal, obs, nfs, ntr, stf_inv, misfit, e->invmat, zeroing, res, l2p, stf, e->st);
    GM_CUDA(cudaGetLastError());
    std::vector<double> l2h(nfs);
    std::vector<double2> stfh(nfs);
    GM_CUDA(cudaMemcpyAsync(l2h.data(), l2p, nfs * sizeof(double), cudaMemcpyDeviceToHost, e->st));
    GM_CUDA(cudaMemcpyAsync(stfh.data(), stf, nfs * sizeof(double2), cudaMemcpyDeviceToHost, e->st));
    GM_CUDA(cudaStreamSynchronize(e->st));
    l2 = 0;
    for (double v : l2h) l2 += v;
    e->last_l2 = 0.5 * l2;
    e->last_l2_each.assign(nf, 0.0);
    for (int i = 0; i < nfs; ++i) e->last_l2_each[i / ns] += 0.5 * l2h[i];
    if (l2_each) {
        l2_each->assign(nf, 0.0);
        for (int i = 0; i < nfs; ++i) (*l2_each)[i / ns] += l2h[i];
    }
    stfu.resize(nfs);
    for (int i = 0; i < nfs; ++i) {
        const double a = std::hypot(stfh[i].x, stfh[i].y);
        stfu[i] = a > 0 ? make_double2(stfh[i].x / a, stfh[i].y / a) : make_double2(1.0, 0.0);
    }
    return GM_OK;
}

}  // namespace

namespace {

// Device bytes per shot of one block solve over the batch: the FP64
// solutions, the working-precision copy, the front update vectors and the
// residual partial sums.
size_t bytes_per_shot(const gm_engine *e) {
    const size_t n = (size_t)e->n, nf = (size_t)e->nf;
    return nf * (n * sizeof(double2) + n * e->csize() + (size_t)e->sym.rhs_total * e->csize() +
                 (size_t)gm::residual_blocks(e->cfg.nx, e->cfg.ny) * 2 * sizeof(double) + 2 * sizeof(double));
}

// Shots per block solve of gm_forward: all of them unless their workspaces
// exceed the device memory left (free now plus what the engine's solve
// workspaces already hold, less a reserve of 5 % of the device and 1 GB),
// or the caller's cap (gm_set_shot_block).
int shot_block(const gm_engine *e, int nshots) {
    const size_t held = e->d_xf.bytes + e->d_t.bytes + e->d_w.bytes + e->d_part.bytes + e->d_norm.bytes;
    const size_t per = std::max<size_t>(1, bytes_per_shot(e));
    if (e->shot_block <= 0 && per * (size_t)nshots <= held) return nshots;   // workspaces in place already
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return nshots;
    const size_t reserve = tot / 20 + ((size_t)1 << 30);
    const size_t avail = fr + held > reserve ? fr + held - reserve : 0;
    size_t blk = avail / per;
    if (e->shot_block > 0) blk = std::min<size_t>(blk, (size_t)e->shot_block);
    return (int)std::max<size_t>(1, std::min<size_t>(blk, (size_t)nshots));
}

}  // namespace

extern "C" int gm_set_shot_block(gm_engine *e, int max_shots) {
    if (!e || max_shots < 0) return fail(GM_ERROR_INVALID, "gm_set_shot_block: bad argument");
    e->shot_block = max_shots;
    return GM_OK;
}

extern "C" int gm_memory_estimate(gm_engine *e, int nmat, size_t *factor_bytes, size_t *shot_bytes) {
    if (!e || nmat <= 0) return fail(GM_ERROR_INVALID, "gm_memory_estimate: bad argument");
    const size_t n = (size_t)e->n, m = (size_t)nmat;
    if (factor_bytes)   // fronts, assembled stencils, mass / stiffness, PML profiles
        *factor_bytes = m * ((size_t)e->sym.front_total * e->csize() + 9 * n * sizeof(double2) + n * sizeof(float2) +
                             n * sizeof(float) + (4 * ((size_t)e->cfg.nx + 2) + 4 * ((size_t)e->cfg.ny + 2)) * 4);
    if (shot_bytes) {
        const int nf = e->nf;
        e->nf = nmat;
        *shot_bytes = bytes_per_shot(e);
        e->nf = nf;
    }
    return GM_OK;
}

extern "C" int gm_forward(gm_engine *e, int nshots, const float *src_x, const float *src_y, int ntr,
                          const int32_t *rec_x, const int32_t *rec_y, float *seis, float *field) {
    int rc = check_ready(e, nshots, ntr);
    if (rc) return rc;
    if (!src_x || !src_y || (ntr > 0 && (!rec_x || !rec_y))) return fail(GM_ERROR_INVALID, "gm_forward: null geometry");
    GM_CUDA(cudaSetDevice(e->device));
    Geometry g;
    if ((rc = make_geometry(e, nshots, src_x, src_y, ntr, rec_x, rec_y, g))) return rc;
    const int blk = shot_block(e, nshots);
    if (blk < nshots) {
        // block solves of at most blk shots each: seismograms and fields are
        // copied out per frequency into the [nf][nshots][...] outputs
        int worst = GM_OK;
        Geometry gb = g;
        for (int s0 = 0; s0 < nshots; s0 += blk) {
            const int nb = std::min(blk, nshots - s0);
            gb.ksrc.assign(g.ksrc.begin() + s0, g.ksrc.begin() + s0 + nb);
            const int brc = forward_and_seis(e, nb, gb, ntr, nullptr);
            if (brc < 0) return brc;
            worst = std::max(worst, brc);
            for (int f = 0; f < e->nf; ++f) {
                if (seis && ntr > 0)
                    GM_CUDA(cudaMemcpyAsync(seis + 2 * ((size_t)f * nshots + s0) * ntr,
                                            e->d_seis.as<float2>() + (size_t)f * nb * ntr,
                                            (size_t)nb * ntr * sizeof(float2), cudaMemcpyDefault, e->st));
            }
            if (field) {
                const size_t cnt = (size_t)e->nf * nb * e->n;
                GM_ALLOC(e->d_field, cnt * sizeof(float2));
                gm::launch_field(e->d_xf.as<double2>(), e->n, e->nf, nb, e->d_field.as<float2>(), e->st);
                GM_CUDA(cudaGetLastError());
                for (int f = 0; f < e->nf; ++f)
                    GM_CUDA(cudaMemcpyAsync(field + 2 * ((size_t)f * nshots + s0) * e->n,
                                            e->d_field.as<float2>() + (size_t)f * nb * e->n,
                                            (size_t)nb * e->n * sizeof(float2), cudaMemcpyDefault, e->st));
            }
            GM_CUDA(cudaStreamSynchronize(e->st));
        }
        e->xf_ns = 0;   // only the last block's solutions are held
        return worst;
    }
    const int solve_rc = forward_and_seis(e, nshots, g, ntr, seis);
    if (solve_rc < 0) return solve_rc;
    if (field) {
        const size_t cnt = (size_t)e->nf * nshots * e->n;
        GM_ALLOC(e->d_field, cnt * sizeof(float2));
        gm::launch_field(e->d_xf.as<double2>(), e->n, e->nf, nshots, e->d_field.as<float2>(), e->st);
        GM_CUDA(cudaGetLastError());
        GM_CUDA(cudaMemcpyAsync(field, e->d_field.p, cnt * sizeof(float2), cudaMemcpyDefault, e->st));
    }
    GM_CUDA(cudaStreamSynchronize(e->st));
    return solve_rc;
}

extern "C" int gm_obj(gm_engine *e, int nshots, const float *src_x, const float *src_y, int ntr,
                      const int32_t *rec_x, const int32_t *rec_y, const float *pobs, int stf_inv, int misfit,
                      float *l2_out) {
    int rc = check_ready(e, nshots, ntr);
    if (rc) return rc;
    if (!pobs || !l2_out || ntr <= 0) return fail(GM_ERROR_INVALID, "gm_obj: need observed data, receivers and an output");
    if (misfit < 1 || misfit > 3) return fail(GM_ERROR_INVALID, "gm_obj: MISFIT must be 1, 2 or 3");
    GM_CUDA(cudaSetDevice(e->device));
    Geometry g;
    if ((rc = make_geometry(e, nshots, src_x, src_y, ntr, rec_x, rec_y, g))) return rc;
    const int solve_rc = forward_and_seis(e, nshots, g, ntr, nullptr);
    if (solve_rc < 0) return solve_rc;
    double l2 = 0;
    std::vector<double2> stfu;
    if ((rc = residuals(e, nshots, ntr, pobs, stf_inv, misfit, l2, stfu))) return rc;
    *l2_out = (float)(0.5 * l2);
    return solve_rc;
}

extern "C" int gm_obj_each(gm_engine *e, int nshots, const float *src_x, const float *src_y, int ntr,
                           const int32_t *rec_x, const int32_t *rec_y, const float *pobs, int stf_inv, int misfit,
                           float *l2_each) {
    int rc = check_ready(e, nshots, ntr);
    if (rc) return rc;
    if (!pobs || !l2_each || ntr <= 0) return fail(GM_ERROR_INVALID, "gm_obj_each: need observed data, receivers and an output");
    if (misfit < 1 || misfit > 3) return fail(GM_ERROR_INVALID, "gm_obj_each: MISFIT must be 1, 2 or 3");
    GM_CUDA(cudaSetDevice(e->device));
    Geometry g;
    if ((rc = make_geometry(e, nshots, src_x, src_y, ntr, rec_x, rec_y, g))) return rc;
    const int solve_rc = forward_and_seis(e, nshots, g, ntr, nullptr);
    if (solve_rc < 0) return solve_rc;
    double l2 = 0;
    std::vector<double2> stfu;
    std::vector<double> each;
    if ((rc = residuals(e, nshots, ntr, pobs, stf_inv, misfit, l2, stfu, &each))) return rc;
    for (int f = 0; f < e->nf; ++f) l2_each[f] = (float)(0.5 * each[f]);
    return solve_rc;
}

namespace {

// Tables of the per-shot gradient taper (gm_set_shot_taper) for
// k_gradient, uploaded into e->d_taper: mode 1 the receivers' product of
// radial coefficients [n] (double), per shot its source window (int4) and
// offset (int), then the windows' coefficients (float); mode 2 the squares'
// mask [n].  Host arithmetic of the reference (host_setup.c).
int shot_taper_tables(gm_engine *e, int ns, const float *sx, const float *sy, int ntr, const int32_t *rx,
                      const int32_t *ry, gm::GradArgs &ga) {
    const gm_config &c = e->cfg;
    const int n = e->n;
    ga.nx = c.nx;
    ga.shot_taper = e->shot_taper;
    if (e->shot_taper == 0) return GM_OK;
    std::vector<unsigned char> host;
    auto put = [&host](const void *p, size_t bytes) {   // 16-byte aligned sections
        const size_t at = (host.size() + 15) / 16 * 16;
        host.resize(at + bytes);
        if (bytes) std::memcpy(host.data() + at, p, bytes);
        return at;
    };
    size_t o_rec = 0, o_win = 0, o_off = 0, o_src = 0, o_mask = 0;
    if (e->shot_taper == 1) {
        std::vector<double> prod(n);
        gmh_srt_receiver_product(c.nx, c.ny, c.dh, e->srt_radius, ntr, rx, ry, prod.data());
        std::vector<int4> win(ns);
        std::vector<int> off(ns);
        std::vector<float> coef;
        for (int s = 0; s < ns; ++s) {
            int x0, x1, y0, y1;
            gmh_srt_range(sx[s], e->srt_radius, c.dh, c.nx, &x0, &x1);
            gmh_srt_range(sy[s], e->srt_radius, c.dh, c.ny, &y0, &y1);
            const int w = std::max(0, x1 - x0 + 1), h = std::max(0, y1 - y0 + 1);
            win[s] = make_int4(x0 - 1, y0 - 1, w, h);
            off[s] = (int)coef.size();
            for (int iy = y0; iy <= y1; ++iy)
                for (int ix = x0; ix <= x1; ++ix) coef.push_back(gmh_srt_coef(ix, iy, c.dh, sx[s], sy[s], e->srt_radius));
        }
        o_rec = put(prod.data(), prod.size() * sizeof(double));
        o_win = put(win.data(), win.size() * sizeof(int4));
        o_off = put(off.data(), off.size() * sizeof(int));
        o_src = put(coef.data(), coef.size() * sizeof(float));
    } else {
        std::vector<unsigned char> mask(n, 0);
        gmh_taper_grad_shot1(c.nx, c.ny, c.dh, e->filtsize, ns, sx, sy, ntr, rx, ry, nullptr, mask.data());
        o_mask = put(mask.data(), mask.size());
    }
    GM_ALLOC(e->d_taper, host.size() + 16);
    GM_CUDA(cudaMemcpyAsync(e->d_taper.p, host.data(), host.size(), cudaMemcpyHostToDevice, e->st));
    GM_CUDA(cudaStreamSynchronize(e->st));   // host is freed on return
    const char *base = static_cast<const char *>(e->d_taper.p);
    if (e->shot_taper == 1) {
        ga.taper_rec = reinterpret_cast<const double *>(base + o_rec);
        ga.taper_win = reinterpret_cast<const int4 *>(base + o_win);
        ga.taper_off = reinterpret_cast<const int *>(base + o_off);
        ga.taper_src = reinterpret_cast<const float *>(base + o_src);
    } else {
        ga.taper_mask = reinterpret_cast<const unsigned char *>(base + o_mask);
    }
    return GM_OK;
}

}  // namespace

extern "C" int gm_set_invmat(gm_engine *e, int invmat) {
    if (!e) return fail(GM_ERROR_INVALID, "gm_set_invmat: no engine");
    if (invmat != 1 && invmat != 2) return fail(GM_ERROR_INVALID, "gm_set_invmat: INVMAT must be 1 (FWI) or 2 (RTM)");
    e->invmat = invmat;
    return GM_OK;
}

extern "C" int gm_set_source_wavelet(gm_engine *e, int nmat, const float *amp) {
    if (!e) return fail(GM_ERROR_INVALID, "gm_set_source_wavelet: no engine");
    if (!amp) {
        e->wavelet.clear();
        return GM_OK;
    }
    if (nmat <= 0) return fail(GM_ERROR_INVALID, "gm_set_source_wavelet: need at least one amplitude");
    for (int i = 0; i < 2 * nmat; ++i)
        if (!std::isfinite(amp[i])) return fail(GM_ERROR_INVALID, "gm_set_source_wavelet: amplitude %d is not finite", i / 2);
    e->wavelet.assign(amp, amp + 2 * (size_t)nmat);
    return GM_OK;
}

extern "C" int gm_set_shot_taper(gm_engine *e, int mode, float srtradius, int filtsize) {
    if (!e) return fail(GM_ERROR_INVALID, "gm_set_shot_taper: no engine");
    if (mode < 0 || mode > 2) return fail(GM_ERROR_INVALID, "gm_set_shot_taper: mode must be 0, 1 or 2");
    if (mode == 1 && !(srtradius > 0.0f)) return fail(GM_ERROR_INVALID, "gm_set_shot_taper: SRTRADIUS must be > 0");
    if (mode == 2 && filtsize < 0) return fail(GM_ERROR_INVALID, "gm_set_shot_taper: FILTSIZE must be >= 0");
    e->shot_taper = mode;
    e->srt_radius = srtradius;
    e->filtsize = filtsize;
    return GM_OK;
}

extern "C" int gm_grad_obj(gm_engine *e, int nshots, const float *src_x, const float *src_y, int ntr,
                           const int32_t *rec_x, const int32_t *rec_y, const float *pobs, int stf_inv, int misfit,
                           float *grad0, float *grad1, float *l2_out, float *seis) {
    int rc = check_ready(e, nshots, ntr);
    if (rc) return rc;
    if (!pobs || ntr <= 0) return fail(GM_ERROR_INVALID, "gm_grad_obj: need observed data and receivers");
    if (misfit < 1 || misfit > 3) return fail(GM_ERROR_INVALID, "gm_grad_obj: MISFIT must be 1, 2 or 3");
    if ((rc = single_model(e, "gm_grad_obj"))) return rc;   // one gradient: one model
    const bool te = e->cfg.physics == GM_PHYS_TE;
    const bool exact = e->cfg.op_mode == GM_OP_EXACT;
    if (exact && (e->cfg.physics != GM_PHYS_AC || stf_inv || misfit != 1 || e->invmat != 1))
        return fail(GM_ERROR_INVALID, "gm_grad_obj: the exact gradient (GM_OP_EXACT) covers acoustic FWI with "
                                      "MISFIT 1, no source estimate and INVMAT 1");
    GM_CUDA(cudaSetDevice(e->device));
    Geometry g;
    if ((rc = make_geometry(e, nshots, src_x, src_y, ntr, rec_x, rec_y, g))) return rc;
    const int nf = e->nf, n = e->n;
    int worst = forward_and_seis(e, nshots, g, ntr, seis);
    if (worst < 0) return worst;
    double l2 = 0;
    std::vector<double2> stfu;
    if ((rc = residuals(e, nshots, ntr, pobs, stf_inv, misfit, l2, stfu))) return rc;

    // adjoint sources and the adjoint solve with the same factors
    if ((rc = upload(e->d_rec_k, g.kadj, e->st))) return rc;
    const size_t cnt = (size_t)nf * nshots * ntr;
    // the reference's adjoint source is conj(res) / DH^2; the exact gradient's is conj(res)
    const double dh2 = exact ? 1.0 : (double)(e->cfg.dh * e->cfg.dh);
    GM_ALLOC(e->d_b, (size_t)nf * n * nshots * sizeof(double2));
    gm::launch_adjoint_src(e->d_b.as<double2>(), n, nf, nshots, ntr, e->d_rec_k.as<int>(), e->d_res.as<double2>() + cnt,
                           dh2, e->st);
    GM_CUDA(cudaGetLastError());
    GM_ALLOC(e->d_xa, (size_t)nf * n * nshots * sizeof(double2));
    // grad_obj_TE.c:149 vs grad_obj_AC.c:147; the exact adjoint solves with M^T
    const int sys = (te || exact) ? GM_SYS_AT : GM_SYS_A;
    gm::RhsPattern pat;   // adjoint sources only at the receivers
    pat.common = g.kadj.data();
    pat.ncommon = ntr;
    const int arc = gm::engine_solve_device(e, sys, nshots, e->d_xa.as<double2>(), e->d_b.as<double2>(), &pat);
    if (arc < 0) return arc;
    e->xa_ns = nshots;
    if (arc > worst) worst = arc;

    // gradient stack + PML frame taper
    if ((rc = ensure_frame(e))) return rc;
    std::vector<double2> om2(nf), om(nf);
    for (int f = 0; f < nf; ++f) {
        float a[2], b[2];
        gmh_gradient_scalars(e->cfg.physics, e->freqs[f], e->cfg.s, a, b);
        if (exact) {   // the derivative of the assembled operator: the assembly's Omega^2
            float o2[2], o[2], o2mu0[2];
            gmh_assembly_scalars(e->cfg.physics, e->freqs[f], e->cfg.s, o2, o, o2mu0);
            a[0] = o2[0];
            a[1] = o2[1];
        }
        om2[f] = make_double2(a[0], a[1]);
        om[f] = make_double2(b[0], b[1]);
    }
    gm::DevBuf scal;
    std::vector<double2> sc;
    sc.insert(sc.end(), stfu.begin(), stfu.end());
    sc.insert(sc.end(), om2.begin(), om2.end());
    sc.insert(sc.end(), om.begin(), om.end());
    if ((rc = upload(scal, sc, e->st))) return rc;
    GM_ALLOC(e->d_grad, 2 * (size_t)n * sizeof(double));
    gm::GradArgs ga{};
    ga.n = n; ga.nf = nf; ga.ns = nshots; ga.te = te;
    ga.xf = e->d_xf.as<double2>(); ga.xa = e->d_xa.as<double2>();
    ga.stfu = scal.as<double2>(); ga.om2 = ga.stfu + stfu.size(); ga.om = ga.om2 + nf;
    ga.m0 = e->d_m0.as<float>() + (size_t)e->models[0] * n; ga.m1 = e->d_m1.as<float>() + (size_t)e->models[0] * n;
    ga.frame = e->d_frame.as<float>(); ga.passes = e->d_frame_pass.as<unsigned char>();
    ga.g0 = e->d_grad.as<double>(); ga.g1 = ga.g0 + n;
    if ((rc = shot_taper_tables(e, nshots, src_x, src_y, ntr, rec_x, rec_y, ga))) return rc;
    if (exact) {
        if (e->shot_taper) return fail(GM_ERROR_INVALID, "gm_grad_obj: the exact gradient takes no per-shot taper");
        float w[6];
        gmh_fd_weights(e->cfg.dh, w);
        gm::launch_gradient_exact(ga, w, e->st);
    } else {
        gm::launch_gradient(ga, e->st);
    }
    GM_CUDA(cudaGetLastError());
    e->last_grad0.resize(n);
    e->last_grad1.assign(te ? n : 0, 0.0);
    GM_CUDA(cudaMemcpyAsync(e->last_grad0.data(), ga.g0, n * sizeof(double), cudaMemcpyDeviceToHost, e->st));
    if (te) GM_CUDA(cudaMemcpyAsync(e->last_grad1.data(), ga.g1, n * sizeof(double), cudaMemcpyDeviceToHost, e->st));
    GM_CUDA(cudaStreamSynchronize(e->st));
    std::vector<float> tmp(n);
    if (grad0) {
        for (int k = 0; k < n; ++k) tmp[k] = (float)e->last_grad0[k];
        GM_CUDA(cudaMemcpy(grad0, tmp.data(), n * sizeof(float), cudaMemcpyDefault));
    }
    if (grad1 && te) {
        for (int k = 0; k < n; ++k) tmp[k] = (float)e->last_grad1[k];
        GM_CUDA(cudaMemcpy(grad1, tmp.data(), n * sizeof(float), cudaMemcpyDefault));
    }
    if (l2_out) *l2_out = (float)(0.5 * l2);
    return worst;
}

extern "C" int gm_get_wavefield_fp64(gm_engine *e, int which, double *x) {
    if (!e || !x || (which != 0 && which != 1)) return fail(GM_ERROR_INVALID, "gm_get_wavefield_fp64: bad argument");
    const int ns = which ? e->xa_ns : e->xf_ns;
    if (ns <= 0) return fail(GM_ERROR_STATE, "gm_get_wavefield_fp64: no %s solution held", which ? "adjoint" : "forward");
    GM_CUDA(cudaSetDevice(e->device));
    const gm::DevBuf &buf = which ? e->d_xa : e->d_xf;
    GM_CUDA(cudaMemcpyAsync(x, buf.p, (size_t)e->nf * e->n * ns * sizeof(double2), cudaMemcpyDefault, e->st));
    GM_CUDA(cudaStreamSynchronize(e->st));
    return GM_OK;
}

extern "C" int gm_get_misfit_fp64(gm_engine *e, int nmat, double *l2, double *l2_each) {
    if (!e) return fail(GM_ERROR_INVALID, "null engine");
    if (e->last_l2_each.empty()) return fail(GM_ERROR_STATE, "no misfit computed yet");
    if (l2_each && nmat != (int)e->last_l2_each.size())
        return fail(GM_ERROR_INVALID, "gm_get_misfit_fp64: the last misfit covered %d matrices, not %d",
                    (int)e->last_l2_each.size(), nmat);
    if (l2) *l2 = e->last_l2;
    if (l2_each) std::memcpy(l2_each, e->last_l2_each.data(), e->last_l2_each.size() * sizeof(double));
    return GM_OK;
}

extern "C" int gm_get_gradient_fp64(gm_engine *e, double *g0, double *g1) {
    if (!e) return fail(GM_ERROR_INVALID, "null engine");
    if (e->last_grad0.empty()) return fail(GM_ERROR_STATE, "no gradient computed yet");
    if (g0) std::memcpy(g0, e->last_grad0.data(), e->last_grad0.size() * sizeof(double));
    if (g1 && !e->last_grad1.empty()) std::memcpy(g1, e->last_grad1.data(), e->last_grad1.size() * sizeof(double));
    return GM_OK;
}

// Diagonal Hessian estimators of the reference, over every shot and every
// factorised frequency:
//   GM_HESS_SHIN   hessian_shin_AC (src/AC/hessian_shin_AC.c:102-132) and
//                  hessian_shin_TE: sum over shots of |J|^2 with
//                  J = 2 Omega^2 F / (rho vp^3) (AC), iOmega F and Omega^2 F (TE);
//   GM_HESS_GREEN  hessian_AC (src/AC/hessian_AC.c:134-165) and hessian_TE:
//                  J also multiplied by the Green's function G_r of every
//                  receiver (a spike at the receiver, RHS_source_AC_hess).
// The reference solves ntr Green's functions for every shot; they do not
// depend on the shot, so here they are solved once per frequency (in blocks
// of receivers) and, since |a F_s G_r|^2 = |a|^2 |F_s|^2 |G_r|^2, the double
// sum over (shot, receiver) is the product of a shot sum and a receiver sum
// per grid point.  Both sums and the result are FP64; the cp_grad_frame
// taper follows (src/AC/hessian_AC.c:174-175).
extern "C" int gm_hessian(gm_engine *e, int mode, int nshots, const float *src_x, const float *src_y, int ntr,
                          const int32_t *rec_x, const int32_t *rec_y, float *hess0, float *hess1) {
    int rc = check_ready(e, nshots, ntr);
    if (rc) return rc;
    if (mode != GM_HESS_SHIN && mode != GM_HESS_GREEN) return fail(GM_ERROR_INVALID, "gm_hessian: unknown mode %d", mode);
    if (mode == GM_HESS_GREEN && ntr <= 0) return fail(GM_ERROR_INVALID, "gm_hessian: GM_HESS_GREEN needs receivers");
    if (e->cfg.physics == GM_PHYS_SH) return fail(GM_ERROR_INVALID, "gm_hessian: the reference has no SH Hessian");
    if ((rc = single_model(e, "gm_hessian"))) return rc;
    const bool te = e->cfg.physics == GM_PHYS_TE;
    GM_CUDA(cudaSetDevice(e->device));
    Geometry g;
    if ((rc = make_geometry(e, nshots, src_x, src_y, mode == GM_HESS_GREEN ? ntr : 0, rec_x, rec_y, g))) return rc;
    const int nf = e->nf, n = e->n;

    // |F|^2 summed over shots.  hessian_shin_TE models its forward fields with
    // RHS_source_AC (src/TE/hessian_shin_TE.c:108), a spike of amplitude
    // 1/DH^2 without the -i Omega mu0 of RHS_source_TE; hessian_TE uses
    // RHS_source_TE (src/TE/hessian_TE.c:113).
    GM_ALLOC(e->d_xf, (size_t)nf * n * nshots * sizeof(double2));
    e->xf_ns = 0;
    e->xa_ns = 0;   // d_xa will hold blocks of receiver Green's functions
    const int src_phys = (te && mode == GM_HESS_SHIN) ? GM_PHYS_AC : e->cfg.physics;
    int worst = forward_solve(e, nshots, g, e->d_xf.as<double2>(), src_phys);
    if (worst < 0) return worst;
    e->xf_ns = nshots;
    gm::DevBuf sq;
    GM_ALLOC(sq, 2 * (size_t)nf * n * sizeof(double));
    double *sqf = sq.as<double>(), *sqg = sqf + (size_t)nf * n;
    gm::launch_hess_sq(e->d_xf.as<double2>(), n, nf, nshots, sqf, 0, e->st);
    GM_CUDA(cudaGetLastError());

    // |G|^2 summed over receivers, the Green's functions solved in blocks
    if (mode == GM_HESS_GREEN) {
        const int blk = std::min(ntr, std::max(nshots, 32));
        const double a = gmh_hess_green_amp(e->cfg.physics, e->cfg.dh);
        std::vector<double2> amp(nf, make_double2(a, 0.0));
        gm::DevBuf amp_buf;
        if ((rc = upload(amp_buf, amp, e->st))) return rc;
        if ((rc = upload(e->d_rec_k, g.kadj, e->st))) return rc;
        GM_ALLOC(e->d_xa, (size_t)nf * n * blk * sizeof(double2));
        for (int r0 = 0; r0 < ntr; r0 += blk) {
            const int nr = std::min(blk, ntr - r0);
            // the reference solves with UMFPACK_A for both physics (src/AC/hessian_AC.c:140, src/TE/hessian_TE.c:140)
            gm::RhsPattern pat;   // one receiver spike per right-hand side
            pat.per_col = g.kadj.data() + r0;
            pat.ncol = nr;
            gm::SpikeRhs sp;
            sp.k = e->d_rec_k.as<int>() + r0;
            sp.amp = amp_buf.as<double2>();
            const int src = gm::engine_solve_device(e, GM_SYS_A, nr, e->d_xa.as<double2>(), nullptr, &pat, &sp);
            if (src < 0) return src;
            if (src > worst) worst = src;
            gm::launch_hess_sq(e->d_xa.as<double2>(), n, nf, nr, sqg, r0 > 0, e->st);
            GM_CUDA(cudaGetLastError());
        }
        GM_CUDA(cudaStreamSynchronize(e->st));   // amp_buf is released on return
    }

    if ((rc = ensure_frame(e))) return rc;
    std::vector<double> w(2 * nf);
    for (int f = 0; f < nf; ++f) {
        float o2[2], o[2];
        gmh_gradient_scalars(e->cfg.physics, e->freqs[f], e->cfg.s, o2, o);
        const double a2 = (double)o2[0] * o2[0] + (double)o2[1] * o2[1];   // |Omega^2|^2
        const double a1 = (double)o[0] * o[0] + (double)o[1] * o[1];       // |Omega|^2 = |i Omega|^2
        w[f] = te ? a1 : 4.0 * a2;                                          // AC: |2 Omega^2|^2
        w[nf + f] = te ? a2 : 0.0;
    }
    gm::DevBuf wbuf;
    if ((rc = upload(wbuf, w, e->st))) return rc;
    GM_ALLOC(e->d_grad, 2 * (size_t)n * sizeof(double));
    GM_ALLOC(e->d_misc, 2 * (size_t)n * sizeof(float));
    gm::HessArgs ha{};
    ha.n = n; ha.nf = nf; ha.te = te;
    ha.sqf = sqf; ha.sqg = mode == GM_HESS_GREEN ? sqg : nullptr;
    ha.w0 = wbuf.as<double>(); ha.w1 = ha.w0 + nf;
    ha.m0 = e->d_m0.as<float>() + (size_t)e->models[0] * n; ha.m1 = e->d_m1.as<float>() + (size_t)e->models[0] * n;
    ha.frame = e->d_frame.as<float>(); ha.passes = e->d_frame_pass.as<unsigned char>();
    ha.h0 = e->d_grad.as<double>(); ha.h1 = ha.h0 + n;
    ha.f0 = e->d_misc.as<float>(); ha.f1 = ha.f0 + n;
    gm::launch_hess_final(ha, e->st);
    GM_CUDA(cudaGetLastError());
    e->last_hess0.resize(n);
    e->last_hess1.assign(te ? n : 0, 0.0);
    GM_CUDA(cudaMemcpyAsync(e->last_hess0.data(), ha.h0, n * sizeof(double), cudaMemcpyDeviceToHost, e->st));
    if (te) GM_CUDA(cudaMemcpyAsync(e->last_hess1.data(), ha.h1, n * sizeof(double), cudaMemcpyDeviceToHost, e->st));
    if (hess0) GM_CUDA(cudaMemcpyAsync(hess0, ha.f0, n * sizeof(float), cudaMemcpyDefault, e->st));
    if (hess1 && te) GM_CUDA(cudaMemcpyAsync(hess1, ha.f1, n * sizeof(float), cudaMemcpyDefault, e->st));
    GM_CUDA(cudaStreamSynchronize(e->st));
    return worst;
}

extern "C" int gm_get_hessian_fp64(gm_engine *e, double *h0, double *h1) {
    if (!e) return fail(GM_ERROR_INVALID, "null engine");
    if (e->last_hess0.empty()) return fail(GM_ERROR_STATE, "no Hessian computed yet");
    if (h0) std::memcpy(h0, e->last_hess0.data(), e->last_hess0.size() * sizeof(double));
    if (h1 && !e->last_hess1.empty()) std::memcpy(h1, e->last_hess1.data(), e->last_hess1.size() * sizeof(double));
    return GM_OK;
}
