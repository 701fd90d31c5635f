/*
 * germaine_gpu.h -- C-ABI of the B200 per-frequency forward/adjoint engine
 * (libgermaine_gpu.so).  Plain pointers and sizes only; every entry point
 * returns an int status (GM_OK = 0, GM_WARNING_* > 0, GM_ERROR_* < 0) that
 * mirrors UMFPACK's convention, and gm_last_error() returns the message of
 * the last failure on the calling thread.
 *
 * Pointer arguments named h_* are host memory; d_* are device memory of the
 * engine's GPU; plain names accept either (copies use unified addressing).
 * Grid arrays are flat row-major [NY][NX] over the FULL grid including the
 * PML frame: grid point (i, j) of the reference (1-based, src/util.c:177
 * NR matrices) is element (j-1)*NX + (i-1).  Complex vectors are
 * interleaved (re, im).  One engine per GPU stream; an engine is not
 * re-entrant.  Every call is synchronous on return unless noted.
 */
#ifndef GERMAINE_GPU_H
#define GERMAINE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (UMFPACK_OK / _WARNING_singular_matrix / _ERROR_*) ---- */
#define GM_OK                     0
#define GM_WARNING_PERTURBED      1  /* pivots were perturbed (tiny or zero pivot) */
#define GM_WARNING_NOT_CONVERGED  2  /* refinement stopped above the residual target */
#define GM_ERROR_OUT_OF_MEMORY   -1
#define GM_ERROR_INVALID         -2  /* bad argument */
#define GM_ERROR_STATE           -3  /* call out of order (e.g. solve before factor) */
#define GM_ERROR_CUDA            -4
#define GM_ERROR_NONFINITE       -5  /* NaN/Inf in the factors or the solution */
#define GM_ERROR_PATTERN         -6  /* matrix is not a 9-point grid pattern (UMFPACK shim) */

/* ---- physics (the reference's PHYSICS, src/germaine.c:86-140) ---- */
#define GM_PHYS_AC 1   /* acoustic pressure: material 0 = vp [m/s], 1 = rho [kg/m^3] */
#define GM_PHYS_SH 2   /* elastic SH: 0 = vs [m/s], 1 = rho [kg/m^3] */
#define GM_PHYS_TE 4   /* EM TE mode: 0 = epsilon [F/m] (absolute), 1 = sigma [S/m] */

/* ---- factor precision ---- */
#define GM_PREC_FP64    0  /* complex128 fronts, FP64 substitution (the drop-in) */
#define GM_PREC_C64_IR  1  /* complex64 fronts + FP64 residual/update refinement */

/* ---- operator orientation ---- */
#define GM_OP_REF   0  /* M = A^T: what UMFPACK factorises after the value
                          overwrite at src/AC/forward_shot_AC.c:41-48 */
#define GM_OP_EXACT 1  /* M = A: the assembled stencil rows; gm_grad_obj then gives
                          the exact discrete gradient of the misfit (acoustic,
                          MISFIT 1, no source estimate): residuals not zeroed,
                          adjoint source conj(res), adjoint solve with M^T, the
                          mass term's 9-point spread of init_A_AC_9p_pml
                          differentiated, no vec2mat shift in the stack */

/* ---- diagonal Hessian estimators (the reference's HESSIAN parameter) ---- */
#define GM_HESS_GREEN 1  /* hessian_AC / hessian_TE: shot and receiver Green's functions */
#define GM_HESS_SHIN  2  /* hessian_shin_AC / hessian_shin_TE (Shin et al. 2001): shots only */

/* ---- solve system (umfpack_zi_solve sys argument) ---- */
#define GM_SYS_A   0   /* M x = b   (UMFPACK_A)   */
#define GM_SYS_AT  1   /* M^T x = b (UMFPACK_Aat, non-conjugate transpose) */

typedef struct gm_engine gm_engine;

/* Grid and discretisation parameters: the reference's .inp globals after
 * forward_AC.c:41-47 (NX, NY already include 2*NPML and NPML+FSSHIFT). */
typedef struct {
    int32_t nx, ny;          /* full grid incl. PML frame */
    float dh;                /* DH [m] */
    int32_t npml;            /* NPML */
    int32_t free_surf;       /* FREE_SURF (FSSHIFT = free_surf ? 0 : npml) */
    float a0_pml;            /* A0_PML */
    float s;                 /* S, Laplace damping */
    int32_t physics;         /* GM_PHYS_* */
    int32_t precision;       /* GM_PREC_* */
    int32_t op_mode;         /* GM_OP_* */
    int32_t leaf_max;        /* nested-dissection leaf size (0 = default 32) */
    double ir_tol;           /* refinement target on max_k ||b_k - M x_k|| / ||b_k|| (0 = 1e-10) */
    int32_t ir_max_iter;     /* refinement iteration cap (0 = default 10) */
    int32_t refine;          /* GM_REFINE_MODE_* (0 = auto) */
    int32_t gmres_restart;   /* GMRES iterations per cycle (0 = default 8, at most 8) */
    int32_t tc_min_block;    /* complex64: contribution blocks of at least this many rows
                                update on the tcgen05 tensor cores (0 = none) */
    double pivot_tol;        /* threshold partial pivoting inside the 32-pivot blocks of
                                every front too large for the small-front kernel: row p
                                is exchanged with the row of largest |entry| in column p
                                (among the block's rows not yet pivoted) when |pivot| <
                                pivot_tol x that entry (0 = default 0.1, UMFPACK's default
                                relative pivot tolerance; < 0 = static pivots only) */
} gm_config;

/* ---- refinement of the solves (gm_config.refine) ---- */
#define GM_REFINE_MODE_AUTO  0  /* iterative refinement; with complex64 factors a matrix whose
                                   last sweep did not contract, or contracted too slowly to
                                   meet the target within the sweeps left (ir_max_iter),
                                   continues with GMRES-IR */
#define GM_REFINE_MODE_IR    1  /* classical iterative refinement only */
#define GM_REFINE_MODE_GMRES 2  /* GMRES-IR for every matrix that needs refinement */

/* Statistics of the last factor/solve (host-side copy). */
typedef struct {
    int64_t n;                  /* unknowns per frequency (NX*NY) */
    int64_t nonzero;            /* NONZERO (src/calc_nonzero.c) */
    int32_t nnodes, nlevels, max_front, max_piv;
    int64_t front_entries;      /* sum nfront^2 per frequency */
    int64_t factor_entries;     /* stored L+U entries per frequency */
    double factor_flops;        /* real flops per frequency (complex FMA = 8) */
    double solve_flops_per_rhs; /* real flops per right-hand side (fwd + bwd) */
    int64_t perturbed_pivots;   /* tiny pivots replaced since the last factor */
    int32_t ir_iterations;      /* refinement sweeps of the last solve */
    double ir_residual;         /* max relative residual after the last solve */
    double ms_assemble, ms_factor, ms_solve, ms_refine;  /* device time of the last calls */
    double ms_subst;            /* device time of the substitutions of the last solve */
    int32_t n_subst;            /* substitutions (initial + refinement) of the last solve */
    int64_t kernel_launches;    /* kernels launched by this library in this process */
    int64_t u_entries;          /* stored U entries (pivot rows) per frequency: the backward pass's factor */
    double ms_subst_bwd;        /* device time of the backward passes of those substitutions */
    int64_t tc_tiles;           /* output tiles of the factorisation routed to tcgen05 */
    int64_t pivot_swaps;        /* row exchanges of the threshold pivoting since the last factor */
} gm_stats;

/* Refinement record of one matrix in the last solve (gm_solve and the solves
 * inside gm_forward, gm_obj, gm_grad_obj -- whose last solve is the adjoint
 * one -- and gm_hessian).  Residuals are max over the matrix's right-hand
 * sides of ||b - M x|| / ||b||, formed in FP64. */
#define GM_REFINE_NONE  0  /* the first (working-precision) solution met the target */
#define GM_REFINE_IR    1  /* classical iterative refinement sweeps */
#define GM_REFINE_GMRES 2  /* GMRES on the correction equation, preconditioned by the factors */
typedef struct {
    double first_residual;   /* residual of the first solution */
    double final_residual;   /* residual on return */
    int32_t sweeps;          /* substitutions after the first one (IR sweeps or GMRES iterations) */
    int32_t method;          /* GM_REFINE_* */
} gm_refine_info;

const char *gm_last_error(void);
int gm_version(void);

/* Create / destroy an engine on CUDA device `device`.  Replaces the
 * per-frequency set-up of forward_shot_AC (src/AC/forward_shot_AC.c:30-35)
 * and umfpack_zi_symbolic (:58): the nested-dissection symbolic analysis
 * of the NX x NY 9-point grid is done once here, on the host, and uploaded. */
int gm_engine_create(int device, const gm_config *cfg, gm_engine **out);
int gm_engine_destroy(gm_engine *e);
int gm_engine_stats(const gm_engine *e, gm_stats *out);
/* The CUDA stream (cudaStream_t) all of the engine's work is issued on, for
 * callers that time or order work against it. */
int gm_engine_stream(const gm_engine *e, void **stream);

/* Material model [NY][NX] (two float arrays, meaning per physics).
 * Replaces readmod()/init_mat_AC (src/AC/init_mat_AC.c:10) input handling. */
int gm_set_model(gm_engine *e, const float *mat0, const float *mat1);

/* nmod material models at once (mat0, mat1: [nmod][NY][NX]) for a batch of
 * matrices from different models: the trial models of a line search, which
 * obj_AC re-assembles and re-factorises one at a time
 * (src/AC/obj_AC.c:10-145, called per trial step by
 * src/AC/parabolicls_AC.c and src/AC/wolfels_AC.c).  gm_set_model is
 * gm_set_models with nmod = 1. */
int gm_set_models(gm_engine *e, int nmod, const float *mat0, const float *mat1);

/* Assemble and factorise the impedance matrices of nfreq frequencies as one
 * batch: init_A_{AC,SH,TE}_9p_pml (src/AC/init_A_AC_9p_pml.c:17) +
 * umfpack_zi_numeric (src/AC/forward_shot_AC.c:61), all frequencies at once.
 * Returns GM_WARNING_PERTURBED if tiny pivots had to be replaced. */
int gm_factor(gm_engine *e, int nfreq, const float *h_freqs);

/* gm_factor over nmat matrices, matrix m assembled at frequency h_freqs[m]
 * from model h_models[m] (NULL: model 0 for all): one level-batched
 * factorisation for every (trial model, frequency) pair.  gm_forward,
 * gm_obj and gm_obj_each then run over all of them; gm_grad_obj requires
 * one model for the whole batch. */
int gm_factor_models(gm_engine *e, int nmat, const float *h_freqs, const int32_t *h_models);

/* Factorise nmat operators given by value instead of assembled from a model:
 * umfpack_zi_numeric (src/AC/forward_shot_AC.c:61) on matrices that arrive
 * as numbers (the UMFPACK shim, libgermaine_umfpack.so, calls this).
 * re/im are [nmat][9][NX*NY] doubles, direction-major in the stencil order
 * NW, N, NE, W, C, E, SW, S, SE (direction q = (di+1) + 3*(dj+1)):
 * entry [m][q][c] is the coefficient that couples grid point c with its
 * neighbour c + di + dj*NX, read in the engine's op_mode -- under GM_OP_REF
 * it is M[c + di + dj*NX][c] (column c of the factorised matrix M), under
 * GM_OP_EXACT M[c][c + di + dj*NX].  Entries whose neighbour lies outside
 * the grid are ignored.  Afterwards gm_solve works as after gm_factor;
 * gm_forward, gm_grad_obj and gm_obj return GM_ERROR_STATE (no model). */
int gm_factor_values(gm_engine *e, int nmat, const double *re, const double *im);

/* Copy the assembled matrix of frequency ifreq out in the reference's
 * triplet layout (row-major, ascending columns; waveAC.Ar/Ai/irow/icol of
 * src/AC/init_A_AC_9p_pml.c:75-80).  Any of the four outputs may be NULL. */
int gm_get_triplets(gm_engine *e, int ifreq, double *Ar, double *Ai, int32_t *irow, int32_t *icol);

/* Autotuner of the substitution's tiles: on the current factors, times one
 * forward and one backward pass over nrhs dense right-hand sides for every
 * candidate tile (32- or 64-row output tiles x 32- or 40-column
 * right-hand-side slices; best of `reps` runs each, 0 = 2) level by level,
 * and keeps per level and pass the fastest.  Solves with nrhs right-hand
 * sides use that table from then on (other counts keep the default
 * rules).  gm_autotune_table returns the tuned right-hand-side count and,
 * for nlevels levels, {forward rows, forward slice/8, backward rows,
 * backward slice/8} per level.  No counterpart in the reference. */
int gm_autotune(gm_engine *e, int nrhs, int reps);
int gm_autotune_table(const gm_engine *e, int *nrhs, int *table, int nlevels);

/* Per-matrix refinement records of the last solve: out[0 .. nmat) for the
 * nmat matrices of the factorised batch (nmat must equal that count).  No
 * counterpart in the reference (UMFPACK's Info array reports one solve); it
 * states, per frequency, the error of the mixed-precision path. */
int gm_refine_report(const gm_engine *e, int nmat, gm_refine_info *out);

/* Solve sys (GM_SYS_A / GM_SYS_AT) for nrhs right-hand sides per frequency
 * with the current factors, followed by FP64 iterative refinement to
 * cfg.ir_tol: umfpack_zi_solve (src/AC/forward_shot_AC.c:88) over a block
 * of right-hand sides.  b and x are [nfreq][N][nrhs] complex128 (interleaved
 * re/im doubles, right-hand side fastest) and must not overlap.  Returns
 * GM_WARNING_NOT_CONVERGED if the target was not met. */
int gm_solve(gm_engine *e, int sys, int nrhs, const double *b, double *x);

/* Forward modelling of all shots of all factorised frequencies
 * (forward_shot_AC, src/AC/forward_shot_AC.c:77-109):
 *   src_x/src_y   [nshots] source coordinates in metres inside the model
 *                 (srcpos[1]/[2], src/sources.c:74-75);
 *   rec_x/rec_y   [ntr] receiver grid indices without the PML offset
 *                 (recpos[1]/[2], src/receiver.c:59-60);
 *   seis          [nfreq][nshots][ntr] complex64 seismograms (precr/preci
 *                 index i + ntr*(ishot-1) + ntr*nshots*(nfreq-1)); may be NULL;
 *   field         [nfreq][nshots][N] complex64 wavefields in the reference's
 *                 vec2mat layout (src/vec2mat.c:19-26, one-slot shift); may be NULL.
 * Sources are spikes of amplitude 1 (AC/SH) or -i*Omega*mu0 (TE) over DH^2. */
int gm_forward(gm_engine *e, int nshots, const float *src_x, const float *src_y,
               int ntr, const int32_t *rec_x, const int32_t *rec_y,
               float *seis, float *field);

/* Memory plan of large problems.  gm_forward solves its shots in blocks
 * when the workspaces of all of them would not fit the device memory left
 * (free memory plus the engine's solve workspaces, less a reserve), or when
 * max_shots > 0 caps the block (0 = memory alone decides); the outputs are
 * the same, and gm_get_wavefield_fp64 then holds no solutions.
 * gm_memory_estimate returns the device bytes of factorising nmat matrices
 * at once and of one shot of a block solve over nmat matrices, so that a
 * caller can choose how many frequencies to factorise together.  No
 * counterpart in the reference (one frequency and one shot at a time). */
int gm_set_shot_block(gm_engine *e, int max_shots);
int gm_memory_estimate(gm_engine *e, int nmat, size_t *factor_bytes, size_t *shot_bytes);

/* Refinement mode (GM_REFINE_MODE_*) and GMRES restart length (0 = the
 * default 8, at most 8) of the following solves: gm_config.refine and
 * gm_config.gmres_restart changed on a live engine.  No counterpart in the
 * reference (its UMFPACK solves are not refined). */
int gm_set_refine(gm_engine *e, int refine, int gmres_restart);

/* FWI objective + gradient of all factorised frequencies (grad_obj_AC,
 * src/AC/grad_obj_AC.c:10-194; grad_obj_TE for GM_PHYS_TE): forward solve,
 * residual (calc_res_AC, MISFIT 1/2/3, optional Wiener source estimate
 * STF_INV), adjoint source, adjoint solve with the same factors
 * (GM_SYS_A for AC as at grad_obj_AC.c:147, GM_SYS_AT for TE as at
 * grad_obj_TE.c:149), gradient stack (ass_grad_AC / ass_grad_TE) and the
 * PML frame taper (cp_grad_frame).
 *   pobs          [nfreq][nshots][ntr] complex64 observed data;
 *   grad0         [NY][NX] AC: vp gradient; TE: sigma gradient (overwritten);
 *   grad1         [NY][NX] TE: epsilon gradient (NULL for AC);
 *   l2            0.5 * sum |res|^2 (the reference's returned L2);
 *   seis          optional modelled seismograms, as in gm_forward. */
int gm_grad_obj(gm_engine *e, int nshots, const float *src_x, const float *src_y,
                int ntr, const int32_t *rec_x, const int32_t *rec_y,
                const float *pobs, int stf_inv, int misfit,
                float *grad0, float *grad1, float *l2, float *seis);

/* INVMAT of calc_res_AC (src/AC/calc_res_AC.c:74-77) for the following
 * gm_grad_obj / gm_obj / gm_obj_each calls: 1 (the default) forms FWI data
 * residuals (MISFIT 1/2/3); 2 makes the residual the observed data itself,
 * the RTM branch that RTM_FD_AC reaches through grad_obj_AC
 * (src/AC/RTM_FD_AC.c:190), so that gm_grad_obj returns the RTM image.
 * The adjoint-source zeroing of tiny observed samples and the misfit sum
 * apply in both modes, as in the reference. */
int gm_set_invmat(gm_engine *e, int invmat);

/* External source wavelet (READ_WAVELET = 1, src/AC/RHS_source_AC.c:40-42,
 * src/TE/RHS_source_TE.c:44-46): amp [nmat][2] holds, per factorised matrix,
 * the complex float amplitude that read_stf_dft returns for its frequency
 * (gm_stf_dft computes it from the SU file); the spikes of gm_forward,
 * gm_obj, gm_obj_each, gm_grad_obj and the forward fields of gm_hessian are
 * then amp / DH^2 instead of 1 / DH^2 (AC, SH) or -i Omega mu0 / DH^2 (TE).
 * nmat must match the batch at solve time (GM_ERROR_STATE otherwise).
 * amp = NULL restores the spike wavelet. */
int gm_set_source_wavelet(gm_engine *e, int nmat, const float *amp);

/* read_stf_dft (src/read_stf_dft.c:12-73) on the host: the SU trace at path
 * (wavelet samples, interval in microseconds for physics <= 3, in
 * nanoseconds for TE) Fourier-transformed at freq, amp[0..1] = real and
 * imaginary part, float results identical to the reference's.  As in the
 * reference the samples enter one place down: the DFT uses samples 1 .. ns-1
 * of the file at times 0, dt, ...; the reference's last term reads one
 * sample past those in the file (whatever its buffer held), taken as 0
 * here.  No GPU needed. */
int gm_stf_dft(const char *path, int physics, float freq, float *amp);

/* Per-shot gradient taper applied by gm_grad_obj inside its shot stack
 * (SWS_TAPER_CIRCULAR_PER_SHOT of ass_grad_AC / ass_grad_TE,
 * src/AC/ass_grad_AC.c:37-43, src/TE/ass_grad_TE.c:41-49):
 *   mode 0  none (the default);
 *   mode 1  taper_grad_shot: each shot's term times the radial taper of
 *           radius srtradius (SRTRADIUS, metres) around its source and
 *           around every receiver;
 *   mode 2  taper_grad_shot1: each shot's term replaced by 1e-5 on the
 *           (2 filtsize + 1)^2 squares (FILTSIZE) around every source of
 *           the call and every receiver.
 * As in the reference, the tapers are centred at the interior source
 * coordinates and receiver indices read as full-grid ones (NPML columns,
 * FSSHIFT rows away from the physical positions).  The product of a
 * shot's coefficients is formed in FP64 and applied to the FP64 term. */
int gm_set_shot_taper(gm_engine *e, int mode, float srtradius, int filtsize);

/* The FP64 solution vectors behind the float outputs: which = 0 the forward
 * wavefields of the last gm_forward / gm_obj / gm_obj_each / gm_grad_obj /
 * gm_hessian call (the umfpack_zi_solve result xr/xi of
 * src/AC/forward_shot_AC.c:88 for every shot), which = 1 the adjoint
 * wavefields of the last gm_grad_obj (src/AC/grad_obj_AC.c:147).  x is
 * [nfreq][N][nshots] complex128 (interleaved re/im, shot fastest) in grid
 * order, before vec2mat's shift.  GM_ERROR_STATE when none is held. */
int gm_get_wavefield_fp64(gm_engine *e, int which, double *x);

/* The last misfit in FP64 before rounding to float: *l2 = 0.5 * sum of
 * |res|^2 over every matrix, shot and receiver of the last gm_obj /
 * gm_obj_each / gm_grad_obj, l2_each[m] the same per matrix (nmat = the
 * batch's matrix count).  Either pointer may be NULL. */
int gm_get_misfit_fp64(gm_engine *e, int nmat, double *l2, double *l2_each);

/* The last gm_grad_obj gradients before rounding to float, in FP64
 * ([NY][NX] each; g1 ignored for AC).  Either pointer may be NULL. */
int gm_get_gradient_fp64(gm_engine *e, double *g0, double *g1);

/* Diagonal of the approximate Hessian over all shots of all factorised
 * frequencies, frame-tapered by cp_grad_frame:
 *   mode GM_HESS_SHIN   hessian_shin_AC (src/AC/hessian_shin_AC.c:48-141) /
 *                       hessian_shin_TE: sum over shots of |J|^2,
 *                       J = 2 Omega^2 F / (rho vp^3) (AC), i Omega F and
 *                       Omega^2 F (TE), F the forward wavefield;
 *   mode GM_HESS_GREEN  hessian_AC (src/AC/hessian_AC.c:48-174) /
 *                       hessian_TE: J further multiplied by the Green's
 *                       function of each receiver (spike source
 *                       RHS_source_AC_hess / RHS_source_TE_hess), summed over
 *                       shots and receivers (rec_x/rec_y as in gm_forward).
 *   hess0  [NY][NX] AC: vp Hessian; TE: sigma Hessian (hess_sigma);
 *   hess1  [NY][NX] TE: epsilon Hessian (NULL for AC).
 * Accumulated in FP64 (gm_get_hessian_fp64), returned as float.  The TE
 * results are not multiplied by MAT1_NORM^2 / MAT2_NORM^2
 * (src/TE/hessian_TE.c:187-188): as for the gradient, the caller scales.
 * One material model for the whole batch; SH has no Hessian in the
 * reference (GM_ERROR_INVALID). */
int gm_hessian(gm_engine *e, int mode, int nshots, const float *src_x, const float *src_y,
               int ntr, const int32_t *rec_x, const int32_t *rec_y, float *hess0, float *hess1);

/* The last gm_hessian results before rounding to float, in FP64. */
int gm_get_hessian_fp64(gm_engine *e, double *h0, double *h1);

/* Objective only (obj_AC, src/AC/obj_AC.c:10-145). */
int gm_obj(gm_engine *e, int nshots, const float *src_x, const float *src_y,
           int ntr, const int32_t *rec_x, const int32_t *rec_y,
           const float *pobs, int stf_inv, int misfit, float *l2);

/* gm_obj with one misfit per factorised matrix: l2_each[m] = 0.5 * the
 * misfit sum of matrix m over its shots (calc_res_AC, src/AC/calc_res_AC.c:
 * 10-95, and the 0.5 L2 of obj_AC, src/AC/obj_AC.c), so that one batched
 * call scores every trial model of a line search.  pobs as for gm_obj,
 * [nmat][nshots][ntr]. */
int gm_obj_each(gm_engine *e, int nshots, const float *src_x, const float *src_y, int ntr, const int32_t *rec_x,
                const int32_t *rec_y, const float *pobs, int stf_inv, int misfit, float *l2_each);

/* Gaussian smoothing of a gradient on the device: gauss_filt
 * (src/gauss_filt.c:10-141), applied by precond() when SPATFILTER = 1
 * (src/precond.c:18).  grad and out are [NY][NX] floats (host or device; out
 * may equal grad); the window follows from VREF, FC_low, FILT_SIZE_GRAD,
 * FILT_SIZE_GRAD1 and DH as in the reference (a size of 0 leaves the
 * gradient unchanged), edges extended by their last value.  Bit-identical
 * to the reference's float result. */
int gm_gauss_filt(int device, int nx, int ny, float dh, float vref, float fc_low, float filt_size_grad,
                  float filt_size_grad1, const float *grad, float *out);

/* The gradient preconditioning of precond() (src/precond.c:10-24) on the
 * GPU, in its order: spatfilter == 1 -> gauss_filt (as gm_gauss_filt);
 * taper_hor != 0 -> taper_grad_hor (src/taper_grad_hor.c:20-31: rows
 * 1 .. GRADT2 + FSSHIFT set to zero, gradt2 = GRADT2); taper != NULL ->
 * taper_grad_file (src/taper_grad_file.c:18-70): the interior multiplied
 * by the NX0 x NY0 taper (x outer, the content of "taper.bin"), the frame
 * filled from the nearest interior column, the top NPML rows from row
 * NPML+1 when free_surf == 1 (which overwrites interior rows, as the
 * reference does) and the bottom rows from the last interior row.
 * Bit-identical; grad [NY][NX] in place, host or device memory. */
int gm_precond(int device, int nx, int ny, int npml, int free_surf, float dh, int spatfilter, float vref,
               float fc_low, float filt_size_grad, float filt_size_grad1, int taper_hor, int gradt2,
               const float *taper, float *grad);

/* Apply the diagonal Hessian to a gradient on the GPU: apply_hess_AC
 * (src/AC/apply_hess_AC.c:11-40), also used for both TE parameters
 * (src/TE/fwi_FD_TE.c:287-288).  MAX_HESS = max |hess| (returned in
 * *max_hess when not NULL), then grad *= 1 / (hess + eps_hess * MAX_HESS)
 * in the reference's float / double arithmetic: bit-identical.  grad and
 * hess are n floats in host or device memory; grad is updated in place. */
int gm_apply_hess(int device, int n, float eps_hess, float *grad, const float *hess, float *max_hess);

/* ---- quasi-Newton l-BFGS on the device ----
 * The reference's l-BFGS update (LBFGS, src/LBFGS.c:12-250; LBFGS_TE,
 * src/TE/LBFGS_TE.c:12, for the two TE classes sigma, epsilon) with its
 * history (y, s of the last m iterations) and the previous gradient and
 * model (what the "<JACOBIAN>_p.old" / "_p_vp.old" files hold) resident on
 * one GPU.  Results are bit-identical to the reference's float arithmetic,
 * including the order of its float dot products (dotp, src/dotp.c).
 * Grids are [nclass][NY][NX] row-major floats in host or device memory;
 * only IDX = IDY = 1 layouts are covered. */
typedef struct gm_lbfgs gm_lbfgs;

/* nclass 1 (AC / SH: NLBFGS_class = 1) or 2 (TE); m = NLBFGS. */
int gm_lbfgs_create(int device, int nx, int ny, int npml, int free_surf, int nclass, int m, gm_lbfgs **out);
int gm_lbfgs_destroy(gm_lbfgs *h);

/* One LBFGS call: first != 0 is the reference's iter == 1 (AC) or
 * LBFGS_RESET == 1 (TE): hgrad = gradm.  Otherwise slot `pointer` (the
 * reference's LBFGS_pointer, 1..m) receives y = grad - previous grad and
 * s = model - previous model, and the two-loop recursion gives hgrad from
 * gradm with the initial Hessian gamma = (y.s)/(y.y) (hess == NULL) or the
 * diagonal Hessian q / (hess + eps_hess * max|hess|) per class (LBFGS_TE
 * with HESSIAN != 0).  hgrad is frame-tapered (cp_grad_frame).  grad and
 * model are kept as the next call's previous gradient and model; model is
 * what the reference saves (AC: vp; TE: sigma / MAT1_NORM and
 * epsilon / MAT2_NORM as scale_grad forms them). */
int gm_lbfgs_step(gm_lbfgs *h, int first, int pointer, const float *grad, const float *gradm,
                  const float *model, const float *hess, float eps_hess, float *hgrad);

/* rot_LBFGS_vec (src/rot_LBFGS_vec.c:10-24): slots 2..m move to 1..m-1. */
int gm_lbfgs_rotate(gm_lbfgs *h);

/* zero_LBFGS / zero_LBFGS1 (src/zero_LBFGS.c): clear the history. */
int gm_lbfgs_zero(gm_lbfgs *h);

/* check_descent (src/check_descent.c:10-31) / check_descent_multi_para_TE:
 * p = -(hgrad . grad) / (grad . grad) with the reference's float sums; the
 * history is cleared when p < 0.  *p receives p (may be NULL). */
int gm_lbfgs_check_descent(gm_lbfgs *h, const float *hgrad, const float *grad, float *p);

/* The previous gradient and model ([nclass][NY][NX]): what the reference's
 * "*.old" files hold (x outer on disk: gm_write_model writes them), so a run
 * can stop and resume. */
int gm_lbfgs_get_old(gm_lbfgs *h, float *grad_old, float *model_old);
int gm_lbfgs_set_old(gm_lbfgs *h, const float *grad_old, const float *model_old);

/* Model update along the search direction: model = model_old + eps_scale *
 * hgrad over n floats, then mode 0 = calc_mat_change_wolfe
 * (src/calc_mat_change_wolfe.c:27-47: values outside [low, up] or below 0
 * keep model_old), mode 1 = calc_mat_change_wolfe_multi_para (clamped to
 * [low, up]).  Bit-identical; host or device buffers. */
int gm_mat_change(int device, int n, int mode, float eps_scale, float low, float up, const float *hgrad,
                  const float *model_old, float *model);

/* Host drop-ins for the reference's per-shot tapers, on one shot's float
 * gradient [NY][NX] (NX, NY with the PML frame) in place, float results
 * identical to the reference's:
 *   gm_taper_grad_shot   taper_grad_shot (src/taper_grad_shot.c:11): the
 *                        radial taper around source ishot (0-based) of
 *                        src_x/src_y (metres, interior coordinates), then
 *                        around every receiver (interior grid indices);
 *   gm_taper_grad_shot1  taper_grad_shot1 (src/taper_grad_shot1.c:11):
 *                        1e-5 on the squares around all nshots sources and
 *                        all receivers, clipped to the grid. */
int gm_taper_grad_shot(int nx, int ny, float dh, float srtradius, int nshots, const float *src_x,
                       const float *src_y, int ntr, const int32_t *rec_x, const int32_t *rec_y, int ishot,
                       float *grad);
int gm_taper_grad_shot1(int nx, int ny, float dh, int filtsize, int nshots, const float *src_x,
                        const float *src_y, int ntr, const int32_t *rec_x, const int32_t *rec_y, float *grad);

/* Host drop-ins for the TE inversion's Tikhonov regularisation on the
 * normalised models (BETA_MAT1 / MAT1_NORM) sigma and (BETA_MAT2 /
 * MAT2_NORM) epsilon, [NY][NX] with the PML frame, float results identical
 * to the reference's:
 *   gm_tikhonov_cost_te  Tikhonov_cost_TE (src/TE/Tikhonov_cost_TE.c:10):
 *                        *l2_out = l2 + LAMBDA_1 * sum 0.5 BETA_MAT1 L(s)^2
 *                        + LAMBDA_2 * sum 0.5 BETA_MAT2 L(e)^2 (l2 when
 *                        both LAMBDAs are <= 0), L the five-point Laplacian
 *                        at every IDX-th / IDY-th interior point;
 *   gm_tikhonov_grad_te  Tikhonov_grad_TE (src/TE/Tikhonov_grad_TE.c:10):
 *                        grad_sigma += LAMBDA_1 BETA_MAT1 L(s),
 *                        grad_epsilon += LAMBDA_2 BETA_MAT2 L(e). */
int gm_tikhonov_cost_te(int nx, int ny, int idx, int idy, float dh, float mat1_norm, float mat2_norm,
                        float beta_mat1, float beta_mat2, float lambda_1, float lambda_2,
                        const float *sigma, const float *epsilon, float l2, float *l2_out);
int gm_tikhonov_grad_te(int nx, int ny, int idx, int idy, float dh, float mat1_norm, float mat2_norm,
                        float beta_mat1, float beta_mat2, float lambda_1, float lambda_2,
                        const float *sigma, const float *epsilon, float *grad_sigma, float *grad_epsilon);

/* ---- the reference's file formats (host stdio, no GPU needed) ---- */
#define GM_SEIS_KEEP_LAST 1  /* gm_write_seis: write the last sample as given */

/* Seismogram file <PICKS_FILE>_p_stage_<n>.bin of write_seis_AC
 * (src/AC/write_seis_AC.c:53-67): float (re, im) pairs, frequency outer,
 * shot, receiver inner -- the [nf][nshots][ntr] layout gm_forward returns.
 * write_seis_AC's gather (src/AC/write_seis_AC.c:43-44) reduces its
 * 1-based arrays from element 0, so the reference always writes the file's
 * LAST sample as 0 + 0i; flags 0 does the same (byte-identical files),
 * GM_SEIS_KEEP_LAST writes that sample as given. */
int gm_write_seis(const char *path, int nf, int nshots, int ntr, int flags, const float *seis);
/* Observed seismograms as read_seis_AC reads them (src/AC/read_seis_AC.c:24-37). */
int gm_read_seis(const char *path, int nf, int nshots, int ntr, float *seis);
/* A [NY][NX] grid without its PML frame, as writemod_true writes models and
 * snapshots (src/writemod_true.c:26-34): interior floats, x outer, every
 * idx-th column and idy-th row (the reference's IDX, IDY). */
int gm_write_model_true(const char *path, int nx, int ny, int npml, int free_surf, int idx, int idy,
                        const float *grid);
/* The full [NY][NX] grid as writemod writes it in binary format 3
 * (src/writemod.c:24-30, src/writedsk.c:32-40): x outer, subsampled. */
int gm_write_model(const char *path, int nx, int ny, int idx, int idy, const float *grid);
/* A full [NY][NX] grid from a file in writemod's layout without
 * subsampling (x outer): the reference's l-BFGS "*.old" files
 * (src/LBFGS.c:183-216, read back at src/LBFGS.c:44-66) and Hessian files
 * (src/AC/hessian_AC.c:178-188) -- so that a run can resume from them. */
int gm_read_grid(const char *path, int nx, int ny, float *grid);
/* One material file as readmod reads it (src/readmod.c:43-104; readmod_SH
 * and readmod_TE alike): interior floats, x outer, placed into the [NY][NX]
 * grid and extended into the PML frame by the nearest interior value. */
int gm_read_model(const char *path, int nx, int ny, int npml, int free_surf, float *grid);

/* gm_solve without device allocation.  No counterpart in the reference: for
 * callers that cannot call cudaMalloc/cudaFree while solving -- cudaFree
 * synchronises the whole device (stalling the caller's own kernels on other
 * streams), and a caller that has reserved its device memory budget up
 * front has none left to give.  Same arguments and result as gm_solve, but
 * b and x must be device (or managed) pointers that do not overlap
 * (GM_ERROR_INVALID otherwise), and every workspace comes from one
 * file-scope device array of 32 MiB; problems whose workspaces do not fit
 * return GM_ERROR_INVALID.  gm_engine_create loads that array (and every
 * kernel this call launches) on the engine's device, where it stays until
 * the process exits, so the call itself allocates nothing.  Calls whose GPU
 * work overlaps race on the shared array.  Each refinement sweep copies the
 * residual norms to the host and waits for the engine's stream, so the call
 * cannot be recorded into a CUDA graph by stream capture.  Statistics:
 * ms_solve and ms_refine are timed, ms_subst is not (0). */
int gm_solve_noalloc(gm_engine *e, int sys, int nrhs, const double *d_b, double *d_x);

/* Batched complex64 GEMM C_i -= A_i * B_i on device pointers: the Schur
 * update of the mixed-precision factorisation (the dense kernel behind
 * umfpack_zi_numeric's front updates) exposed for testing.  dims holds
 * (m, n, k, lda, ldb, ldc) per problem, all matrices column-major.
 * backend 1 = tcgen05 tensor cores (3xTF32 split products), 0 = CUDA cores. */
int gm_cgemm_sub_c64(int device, int backend, int nprob, const int32_t *dims, void *const *A, void *const *B,
                     void *const *C);

/* Failure-path check of the tensor-core kernels' bounded waits: one CTA
 * waits, with the same bounded mbarrier wait as the tcgen05 kernels, on an
 * mbarrier that nothing signals; the wait gives up after `polls` polls
 * (1 .. 2^24) and *timed_out is set to 1 (0 would mean the wait returned
 * without its phase completing).  Where a tcgen05 kernel's wait runs out it
 * sets an error flag that the factorisation returns as GM_ERROR_CUDA
 * instead of hanging.  No counterpart in the reference. */
int gm_wait_probe(int device, long long polls, int *timed_out);

/* Measured FP64 FMA throughput of the device's CUDA cores in TFLOP/s (a DFMA
 * chain kernel timed with CUDA events, best of four launches after two
 * warm-up launches): the denominator of the FP64 roofline fractions.  No
 * counterpart in the reference. */
int gm_peak_fp64(int device, double *tflops);
/* The same for FP64 matrix instructions (mma.sync m8n8k4 f64). */
int gm_peak_fp64_mma(int device, double *tflops);

/* ---- symbolic-analysis introspection (host only, no GPU needed) ---- */
typedef struct gm_symbolic gm_symbolic;
int gm_symbolic_create(int nx, int ny, int leaf_max, gm_symbolic **out);
int gm_symbolic_destroy(gm_symbolic *s);
/* sizes[0..15]: n, nnodes, nlevels, nvars, front_total, ninv, nent, rhs_total,
 * factor_entries, max_front, max_piv, 0... */
int gm_symbolic_sizes(const gm_symbolic *s, int64_t *sizes);
/* what: 0 perm, 1 iperm, 2 npiv, 3 nfront, 4 parent, 5 height, 6 child0,
 * 7 child1, 8 var_off(int64), 9 vars, 10 front_off(int64), 11 inv_off(int64),
 * 12 inv, 13 ent_off(int64), 14 ent_pos, 15 ent_id, 16 rhs_off(int64),
 * 17 lvl_off, 18 lvl_nodes */
int gm_symbolic_export(const gm_symbolic *s, int what, void *dst);
double gm_symbolic_flops(const gm_symbolic *s, int which /* 0 factor, 1 solve per rhs */);

#ifdef __cplusplus
}
#endif
#endif
