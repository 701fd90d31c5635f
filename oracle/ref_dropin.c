/*
 * oracle/ref_dropin.c -- TEST INFRASTRUCTURE ONLY (never shipped, never
 * measured as the product).
 *
 * Entry points that run the reference's UNMODIFIED per-frequency drivers
 *   forward_shot_AC   src/AC/forward_shot_AC.c:10
 *   grad_obj_AC       src/AC/grad_obj_AC.c:10
 *   hessian_shin_AC   src/AC/hessian_shin_AC.c:10   (HESSIAN = 2)
 *   hessian_AC        src/AC/hessian_AC.c:10        (HESSIAN = 1)
 *   hessian_shin_TE   src/TE/hessian_shin_TE.c:10
 *   hessian_TE        src/TE/hessian_TE.c:10
 * compiled from the reference tree against include/germaine_umfpack.h (as
 * "umfpack.h") and linked with libgermaine_umfpack.so, so that every
 * UMFPACK call of the drivers lands on the GPU engine.  oracle/Makefile
 * builds this file, oracle/ref_harness.c and the drivers' dependencies into
 * oracle/_ref/libgermaine_ref_dropin.so.  This file contains no reference
 * code: it fills the drivers' structs and globals (include/fd.h,
 * include/globvar.h) from flat arrays and copies the results out.
 * ref_set_grid (ref_harness.c) must be called first.
 */
#include "fd.h"

/* the reference's globals (defined by include/globvar.h in ref_harness.c) */
extern int NX, NY, NXNY, NONZERO, NSHOT1, NSHOT2, NSHOTS, NF, SNAP, SEISMO, INFO, READ_REC, MYID, NP;
extern int N_STREAMER, STF_INV, MISFIT, INVMAT, NFREQ1, NFREQ2;
extern float MAT1_NORM, MAT2_NORM;
extern char JACOBIAN[STRING_SIZE];

/* the drivers' prototypes not declared in fd.h */
void pml_pro(struct PML_AC *PML_AC, struct waveAC *waveAC);

static float **nr_from_flat(const float *flat)
{
    float **m = matrix(0, NY + 1, 0, NX + 1);
    int i, j;
    for (j = 1; j <= NY; j++)
        for (i = 1; i <= NX; i++) m[j][i] = flat[(j - 1) * NX + (i - 1)];
    return m;
}

static void alloc_wave(struct waveAC *w, struct PML_AC *p, struct matAC *m, const float *vp, const float *rho)
{
    p->dampxr = vector(0, NX + 1); p->dampxi = vector(0, NX + 1);
    p->dampxhr = vector(0, NX + 1); p->dampxhi = vector(0, NX + 1);
    p->dampyr = vector(0, NY + 1); p->dampyi = vector(0, NY + 1);
    p->dampyhr = vector(0, NY + 1); p->dampyhi = vector(0, NY + 1);
    m->vp = nr_from_flat(vp); m->rho = nr_from_flat(rho);
    m->ivp2 = matrix(0, NY + 1, 0, NX + 1); m->b = matrix(0, NY + 1, 0, NX + 1);
    w->pr = matrix(0, NY + 1, 0, NX + 1); w->pi = matrix(0, NY + 1, 0, NX + 1);
    w->RHSr = calloc((size_t)NXNY + 1, sizeof(double));
    w->RHSi = calloc((size_t)NXNY + 1, sizeof(double));
    w->Ar = calloc((size_t)NONZERO, sizeof(double));
    w->Ai = calloc((size_t)NONZERO, sizeof(double));
    w->irow = calloc((size_t)NONZERO, sizeof(int));
    w->icol = calloc((size_t)NONZERO, sizeof(int));
}

static void free_wave(struct waveAC *w, struct PML_AC *p, struct matAC *m)
{
    free_vector(p->dampxr, 0, NX + 1); free_vector(p->dampxi, 0, NX + 1);
    free_vector(p->dampxhr, 0, NX + 1); free_vector(p->dampxhi, 0, NX + 1);
    free_vector(p->dampyr, 0, NY + 1); free_vector(p->dampyi, 0, NY + 1);
    free_vector(p->dampyhr, 0, NY + 1); free_vector(p->dampyhi, 0, NY + 1);
    free_matrix(m->vp, 0, NY + 1, 0, NX + 1); free_matrix(m->rho, 0, NY + 1, 0, NX + 1);
    free_matrix(m->ivp2, 0, NY + 1, 0, NX + 1); free_matrix(m->b, 0, NY + 1, 0, NX + 1);
    free_matrix(w->pr, 0, NY + 1, 0, NX + 1); free_matrix(w->pi, 0, NY + 1, 0, NX + 1);
    free(w->RHSr); free(w->RHSi); free(w->Ar); free(w->Ai); free(w->irow); free(w->icol);
}

static float **srcpos_nr(int nshots, const float *sx, const float *sy)
{
    float **s = matrix(1, 8, 1, nshots);
    int k;
    for (k = 1; k <= nshots; k++) { s[1][k] = sx[k - 1]; s[2][k] = sy[k - 1]; }
    return s;
}

static int **recpos_nr(int ntr, const int *rx, const int *ry)
{
    int **r = imatrix(1, 3, 1, ntr), t;
    for (t = 1; t <= ntr; t++) { r[1][t] = rx[t - 1]; r[2][t] = ry[t - 1]; r[3][t] = 0; }
    return r;
}

static void driver_globals(int nshots, int nf)
{
    NSHOT1 = 1; NSHOT2 = nshots + 1; NSHOTS = nshots; NF = nf;
    SNAP = 0; INFO = 0; READ_REC = 0; MYID = 0; NP = 1; N_STREAMER = 0;
}

/* forward_shot_AC for one frequency (its call from forward_AC.c:167 after
 * pml_pro and init_mat_AC): seismograms [nshots][ntr] into precr/preci. */
void dropin_forward_shot_ac(float freq, const float *vp, const float *rho, int nshots, const float *sx,
                            const float *sy, int ntr, const int *rx, const int *ry, float *precr, float *preci)
{
    struct waveAC w; struct PML_AC p; struct matAC m;
    float **srcpos;
    driver_globals(nshots, 1);
    SEISMO = 1;
    alloc_wave(&w, &p, &m, vp, rho);
    w.freq = freq;
    w.precr = precr - 1; w.preci = preci - 1;
    srcpos = srcpos_nr(nshots, sx, sy);
    acq.recpos = recpos_nr(ntr, rx, ry);
    pml_pro(&p, &w);
    init_mat_AC(&w, &m);
    forward_shot_AC(&w, &p, &m, srcpos, nshots, acq.recpos, ntr, 1, 1);
    free_imatrix(acq.recpos, 1, 3, 1, ntr);
    free_matrix(srcpos, 1, 8, 1, nshots);
    free_wave(&w, &p, &m);
}

/* INVMAT for the next dropin_grad_obj_ac calls: 1 FWI (default), 2 RTM
 * (calc_res_AC takes the observed data as residual, as under RTM_FD_AC). */
static int dropin_invmat = 1;
void dropin_set_invmat(int invmat) { dropin_invmat = invmat; }

/* grad_obj_AC over the frequencies freqs[0..nf) (one stage): observed data
 * pobs and modelled data prec are [nf][nshots][ntr]; the frame-tapered
 * gradient (NY x NX, row-major) goes to grad, the objective is returned. */
float dropin_grad_obj_ac(int nf, const float *freqs, const float *vp, const float *rho, int nshots,
                         const float *sx, const float *sy, int ntr, const int *rx, const int *ry,
                         const float *pobsr, const float *pobsi, int stf_inv, int misfit, float *grad)
{
    struct waveAC w; struct PML_AC p; struct matAC m; struct fwiAC f;
    float **srcpos, l2, *precr, *preci, *stage;
    int i, j;
    driver_globals(nshots, nf);
    STF_INV = stf_inv; MISFIT = misfit; INVMAT = dropin_invmat;
    NFREQ1 = 1; NFREQ2 = nf + 1;
    alloc_wave(&w, &p, &m, vp, rho);
    precr = calloc((size_t)nf * nshots * ntr, sizeof(float));
    preci = calloc((size_t)nf * nshots * ntr, sizeof(float));
    stage = malloc(sizeof(float) * (size_t)nf);
    for (i = 0; i < nf; i++) stage[i] = freqs[i];
    w.stage_freq = stage - 1;
    w.precr = precr - 1; w.preci = preci - 1;
    w.pobsr = (float *)pobsr - 1; w.pobsi = (float *)pobsi - 1;
    w.presr = vector(1, ntr); w.presi = vector(1, ntr);
    f.grad = matrix(1, NY, 1, NX);
    f.forwardr = matrix(1, NY, 1, NX); f.forwardi = matrix(1, NY, 1, NX);
    srcpos = srcpos_nr(nshots, sx, sy);
    acq.recpos = recpos_nr(ntr, rx, ry);
    l2 = grad_obj_AC(&f, &w, &p, &m, srcpos, nshots, acq.recpos, ntr, 1, 1);
    for (j = 1; j <= NY; j++)
        for (i = 1; i <= NX; i++) grad[(j - 1) * NX + (i - 1)] = f.grad[j][i];
    free_imatrix(acq.recpos, 1, 3, 1, ntr);
    free_matrix(srcpos, 1, 8, 1, nshots);
    free_matrix(f.grad, 1, NY, 1, NX);
    free_matrix(f.forwardr, 1, NY, 1, NX); free_matrix(f.forwardi, 1, NY, 1, NX);
    free_vector(w.presr, 1, ntr); free_vector(w.presi, 1, ntr);
    free(stage); free(precr); free(preci);
    free_wave(&w, &p, &m);
    return l2;
}

static void flat_from_nr(float **m, float *flat)
{
    int i, j;
    for (j = 1; j <= NY; j++)
        for (i = 1; i <= NX; i++) flat[(j - 1) * NX + (i - 1)] = m[j][i];
}

static float *stage_freqs(struct waveAC *w, int nf, const float *freqs)
{
    float *stage = malloc(sizeof(float) * (size_t)nf);
    int i;
    for (i = 0; i < nf; i++) stage[i] = freqs[i];
    w->stage_freq = stage - 1;
    NFREQ1 = 1; NFREQ2 = nf + 1;
    return stage;
}

/* hessian_shin_AC (mode 2) or hessian_AC (mode 1) over freqs[0..nf): the
 * frame-tapered Hessian (NY x NX) into hess; the drivers also write
 * <jacobian>_hess (float, x outer). */
void dropin_hessian_ac(int mode, int nf, const float *freqs, const float *vp, const float *rho, int nshots,
                       const float *sx, const float *sy, int ntr, const int *rx, const int *ry, const char *jacobian,
                       float *hess)
{
    struct waveAC w; struct PML_AC p; struct matAC m; struct fwiAC f;
    float **srcpos, *stage;
    driver_globals(nshots, nf);
    snprintf(JACOBIAN, STRING_SIZE, "%s", jacobian);
    alloc_wave(&w, &p, &m, vp, rho);
    stage = stage_freqs(&w, nf, freqs);
    f.hess = matrix(1, NY, 1, NX);
    f.forwardr = matrix(1, NY, 1, NX); f.forwardi = matrix(1, NY, 1, NX);
    srcpos = srcpos_nr(nshots, sx, sy);
    acq.recpos = recpos_nr(ntr, rx, ry);
    if (mode == 2) hessian_shin_AC(&f, &w, &p, &m, srcpos, nshots, acq.recpos, ntr, 1, 1);
    else hessian_AC(&f, &w, &p, &m, srcpos, nshots, acq.recpos, ntr, 1, 1);
    flat_from_nr(f.hess, hess);
    free_imatrix(acq.recpos, 1, 3, 1, ntr);
    free_matrix(srcpos, 1, 8, 1, nshots);
    free_matrix(f.hess, 1, NY, 1, NX);
    free_matrix(f.forwardr, 1, NY, 1, NX); free_matrix(f.forwardi, 1, NY, 1, NX);
    free(stage);
    free_wave(&w, &p, &m);
}

/* hessian_shin_TE (mode 2) or hessian_TE (mode 1) with MAT1_NORM =
 * MAT2_NORM = 1: hess_sigma, hess_epsilon (NY x NX); the drivers also write
 * <jacobian>_hess_sigma and <jacobian>_hess_epsilon. */
void dropin_hessian_te(int mode, int nf, const float *freqs, const float *eps, const float *sig, int nshots,
                       const float *sx, const float *sy, int ntr, const int *rx, const int *ry, const char *jacobian,
                       float *hess_sigma, float *hess_epsilon)
{
    struct waveAC w; struct PML_AC p; struct matAC unused; struct matTE m; struct fwiTE f;
    float **srcpos, *stage;
    driver_globals(nshots, nf);
    snprintf(JACOBIAN, STRING_SIZE, "%s", jacobian);
    MAT1_NORM = 1.0f; MAT2_NORM = 1.0f;
    alloc_wave(&w, &p, &unused, eps, sig);   /* the AC material grids are not read by the TE drivers */
    m.epsilon = nr_from_flat(eps); m.sigma = nr_from_flat(sig);
    stage = stage_freqs(&w, nf, freqs);
    f.hess_sigma = matrix(1, NY, 1, NX); f.hess_epsilon = matrix(1, NY, 1, NX);
    f.forwardr = matrix(1, NY, 1, NX); f.forwardi = matrix(1, NY, 1, NX);
    srcpos = srcpos_nr(nshots, sx, sy);
    acq.recpos = recpos_nr(ntr, rx, ry);
    if (mode == 2) hessian_shin_TE(&f, &w, &p, &m, srcpos, nshots, acq.recpos, ntr, 1, 1);
    else hessian_TE(&f, &w, &p, &m, srcpos, nshots, acq.recpos, ntr, 1, 1);
    flat_from_nr(f.hess_sigma, hess_sigma);
    flat_from_nr(f.hess_epsilon, hess_epsilon);
    free_imatrix(acq.recpos, 1, 3, 1, ntr);
    free_matrix(srcpos, 1, 8, 1, nshots);
    free_matrix(f.hess_sigma, 1, NY, 1, NX); free_matrix(f.hess_epsilon, 1, NY, 1, NX);
    free_matrix(f.forwardr, 1, NY, 1, NX); free_matrix(f.forwardi, 1, NY, 1, NX);
    free_matrix(m.epsilon, 0, NY + 1, 0, NX + 1); free_matrix(m.sigma, 0, NY + 1, 0, NX + 1);
    free(stage);
    free_wave(&w, &p, &unused);
}
