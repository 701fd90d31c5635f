// Engine state behind the gm_engine handle.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/germaine_gpu.h"
#include "common.hpp"
#include "kernels.cuh"
#include "symbolic.hpp"

namespace gm {

// Owning device allocation.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t nb) {  // grow-only
        if (nb <= bytes && p) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, nb ? nb : 16);
        if (e == cudaSuccess) {
            bytes = nb;
        } else {
            p = nullptr;
            (void)cudaGetLastError();   // reported through the return value, not left for later checks
        }
        return e;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

}  // namespace gm

struct gm_engine {
    int device = 0;
    cudaStream_t st = nullptr;
    gm_config cfg{};
    int fsshift = 0;
    int n = 0;
    gm::Symbolic sym;

    // device copy of the symbolic structure
    gm::DevBuf d_npiv, d_nfront, d_child0, d_child1, d_vars, d_inv, d_lvl_nodes;
    gm::DevBuf d_front_off, d_var_off, d_inv_off, d_rhs_off;
    gm::DevBuf d_ent_dst, d_ent_src, d_ent_lvl_off;
    std::vector<gm::LevelInfo> levels;
    gm::DevSym dsym{};

    // model
    gm::DevBuf d_m0, d_m1, d_stiff;  // models [nmod][n]; stiffness per matrix [nf][n]
    int nmod = 0;
    bool have_model = false;

    // factorisation of the current frequency batch
    int nf = 0;
    std::vector<float> freqs;
    std::vector<int> models;    // material model of each matrix of the batch
    gm::DevBuf d_A, d_mass, d_pml, d_fq, d_front, d_npert, d_amax;
    // threshold pivoting record [nf][n] (FactorArgs::pivsrc): every slot up
    // to pivsrc_ready_nf of the buffer at pivsrc_ready holds the identity
    // outside the pivoted levels
    gm::DevBuf d_pivsrc;
    const void *pivsrc_ready = nullptr;
    int pivsrc_ready_nf = 0;
    bool factored = false;
    bool values_only = false;   // operator given by gm_factor_values (no frequencies / model)

    // contribution-block GEMM plan per level (rebuilt when the front
    // storage moves or the batch size changes)
    struct CbPlan { int backend; int64_t prob_off, tile_off; int ntiles; };
    std::vector<CbPlan> cb_plan;
    gm::DevBuf d_cb_probs, d_cb_tiles, d_tcerr;
    const void *cb_plan_base = nullptr;
    int cb_plan_nf = 0;
    // the factorisation's launch sequence as a CUDA graph, replayed while
    // the buffers and the batch it was captured for stay the same
    struct FactorGraphKey {
        const void *front = nullptr, *A = nullptr, *amax = nullptr, *npert = nullptr, *tcerr = nullptr;
        const void *probs = nullptr, *tiles = nullptr, *pivsrc = nullptr;
        int nf = 0, fp64 = 0;
        bool operator==(const FactorGraphKey &o) const {
            return front == o.front && A == o.A && amax == o.amax && npert == o.npert && tcerr == o.tcerr &&
                   probs == o.probs && tiles == o.tiles && pivsrc == o.pivsrc && nf == o.nf && fp64 == o.fp64;
        }
    };
    FactorGraphKey fgraph_key, fgraph_seen;
    cudaGraphExec_t fgraph = nullptr;
    long long fgraph_kernels = 0;
    bool fgraph_broken = false;   // capture failed once: launch directly

    // solve workspaces
    gm::DevBuf d_x, d_b, d_r, d_t, d_w, d_part, d_norm;
    gm::DevBuf d_fmap;                          // matrices still refined (device list)
    // GMRES-IR: Krylov vectors [m+1][ng][n][nrhs] c128, preconditioned
    // vectors [m][ng][n][nrhs] (working precision), reductions, coefficients
    gm::DevBuf d_gv, d_gz, d_gpart, d_gnorm, d_gcoef, d_gmap;
    std::vector<int> h_fmap;                    // its host copy (kept alive for async uploads)
    std::vector<gm_refine_info> refine_info;    // per matrix, of the last solve

    // epilogue state
    gm::DevBuf d_src_k, d_rec_k, d_seis, d_field, d_res, d_grad, d_frame, d_frame_pass, d_misc;
    gm::DevBuf d_xf, d_xa;   // forward / adjoint solutions kept for the gradient
    int xf_ns = 0, xa_ns = 0; // right-hand sides held in d_xf / d_xa (0: none valid)
    gm::DevBuf d_mask;       // forward-pass pruning mask of the current solve
    gm::DevBuf d_work;       // its live (front position, slice) pairs per level
    // substitution tiles per level chosen by gm_autotune for tuned_nrhs
    // right-hand sides and this precision: {fwd rt, fwd B, bwd rt, bwd B}
    std::vector<int> lvl_cfg;
    int tuned_nrhs = 0;
    std::vector<int> work_off;
    std::vector<int> work_w; // per level: slice width the pairs were built for
    bool have_work = false;
    std::vector<double> last_grad0, last_grad1;
    // per-shot gradient taper of ass_grad (SWS_TAPER_CIRCULAR_PER_SHOT 0, 1, 2),
    // its radius (SRTRADIUS, metres) and square half-width (FILTSIZE)
    int invmat = 1;               // INVMAT of calc_res_AC: 1 FWI residuals, 2 RTM (observed data)
    int shot_block = 0;           // gm_forward's cap on shots per block solve (0: memory decides)
    double last_l2 = 0;           // 0.5 * misfit sum of the last gm_obj / gm_obj_each / gm_grad_obj, FP64
    std::vector<double> last_l2_each;   // the same per matrix
    std::vector<float> wavelet;   // [nf][2] source amplitudes of READ_WAVELET = 1 (empty: spikes)
    int shot_taper = 0;
    float srt_radius = 0.0f;
    int filtsize = 0;
    gm::DevBuf d_taper;   // the taper's tables for the gradient kernel
    std::vector<double> last_hess0, last_hess1;

    gm_stats stats{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_s0 = nullptr, ev_s1 = nullptr, ev_sm = nullptr;

    gm_engine() = default;
    gm_engine(const gm_engine &) = delete;
    gm_engine &operator=(const gm_engine &) = delete;
    ~gm_engine() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_s0) cudaEventDestroy(ev_s0);
        if (ev_s1) cudaEventDestroy(ev_s1);
        if (ev_sm) cudaEventDestroy(ev_sm);
        if (fgraph) cudaGraphExecDestroy(fgraph);
        if (st) cudaStreamDestroy(st);
    }

    size_t csize() const { return cfg.precision == GM_PREC_FP64 ? sizeof(double2) : sizeof(float2); }
};

namespace gm {
// Where the right-hand sides can be nonzero (for pruning the forward pass of
// the first substitution): right-hand side r is nonzero at most on row
// per_col[r] (a spike; -1: none) and on the rows in `common`.  Rows are grid
// indices.  A solve given no pattern treats every right-hand side as dense.
struct RhsPattern {
    const int *per_col = nullptr;
    int ncol = 0;
    const int *common = nullptr;
    int ncommon = 0;
};

// Spike right-hand sides given implicitly (device arrays): right-hand side r
// of frequency f is amp[f] at row k[r] and zero elsewhere, so no dense b is
// formed, copied or read.
struct SpikeRhs {
    const int *k = nullptr;         // [nrhs]
    const double2 *amp = nullptr;   // [nf]
};

// once per device at engine creation: the scratch array and kernels of
// gm_solve_noalloc (noalloc.cu)
int noalloc_prepare(int device);

// internal entry points shared between translation units
int engine_solve_device(gm_engine *e, int sys, int nrhs, double2 *d_x_out, const double2 *d_b_in,
                        const RhsPattern *pattern = nullptr, const SpikeRhs *spikes = nullptr);
}
