/*
 * oracle/port.c -- TEST ORACLE (CPU restatement).  Only tests/, the smoke
 * check and bench.py's cpu_baseline leg load this file's library, and only
 * as the checker: it is never the product path.
 *
 * Plain-C restatement of GERMAINE's per-frequency hot-path arithmetic on
 * flat, 0-based, row-major [NY][NX] arrays (grid point (i, j), 1-based in
 * the reference, is flat index (j-1)*NX + (i-1)).  Every function cites the
 * reference file:line it follows.  Floating-point types and evaluation order
 * follow the reference exactly (complex float terms promoted to complex
 * double where a double literal appears), so a gcc build without FMA
 * reproduces the reference's roundings bit for bit; the pin is
 * tests/test_oracle_pin.py against the reference's own sources compiled
 * into oracle/_ref and against the committed fixtures in tests/golden/.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct {
    int nx, ny, npml, free_surf, fsshift;
    float dh, a0_pml, s;
} port_grid;

static int iround_f(float x) { return (int)floor(x + 0.5); } /* fd.h:20 */

/* NONZERO of the 9-point pattern, closed form of src/calc_nonzero.c:10-52 */
int port_nonzero(int nx, int ny) { return 9 * nx * ny - 6 * nx - 6 * ny + 4; }

/* PML stretch profiles, src/pml_pro.c:20-160.  out = 8 arrays: x-node r/i,
 * x-half r/i (NX+2 each), then y-node r/i, y-half r/i (NY+2 each). */
void port_pml(const port_grid *g, float freq, float *out)
{
    const int nxa = g->nx + 2, nya = g->ny + 2;
    float *xr = out, *xi = out + nxa, *xhr = out + 2 * nxa, *xhi = out + 3 * nxa;
    float *yr = out + 4 * nxa, *yi = yr + nya, *yhr = yr + 2 * nya, *yhi = yr + 3 * nya;
    const float halfpi = M_PI / 2.0;
    const complex float ci = 0.0 + 1.0 * I;
    const float lpml = g->npml * g->dh;
    const complex float om = 2.0 * M_PI * (freq - I * g->s);
    for (int k = 0; k < nxa; k++) { xr[k] = 1.0f; xi[k] = 0.0f; xhr[k] = 1.0f; xhi[k] = 0.0f; }
    for (int k = 0; k < nya; k++) { yr[k] = 1.0f; yi[k] = 0.0f; yhr[k] = 1.0f; yhi[k] = 0.0f; }
    for (int p = 1; p <= g->npml; p++) {
        float x = p * g->dh;
        float xh = x + 0.5 * g->dh;
        float prof = g->a0_pml * (1.0 - cos((lpml - x) * halfpi / lpml));
        float profh = g->a0_pml * (1.0 - cos((lpml - xh) * halfpi / lpml));
        complex double sn = 1.0 / (1.0 + prof / (ci * om));
        complex double sh = 1.0 / (1.0 + profh / (ci * om));
        xr[p] = creal(sn); xi[p] = cimag(sn); xhr[p] = creal(sh); xhi[p] = cimag(sh);
        yr[p] = xr[p]; yi[p] = xi[p]; yhr[p] = xhr[p]; yhi[p] = xhi[p];
        xr[g->nx - p + 1] = xr[p]; xi[g->nx - p + 1] = xi[p];
        xhr[g->nx - p + 1] = xhr[p]; xhi[g->nx - p + 1] = xhi[p];
        yr[g->ny - p + 1] = xr[p]; yi[g->ny - p + 1] = xi[p];
        yhr[g->ny - p + 1] = xhr[p]; yhi[g->ny - p + 1] = xhi[p];
        if (g->free_surf == 1) { yr[p] = 1.0f; yi[p] = 0.0f; yhr[p] = 1.0f; yhi[p] = 0.0f; }
    }
    xr[0] = xr[1]; xi[0] = xi[1]; xhr[0] = xhr[1]; xhi[0] = xhi[1];
    xr[g->nx + 1] = xr[g->nx]; xi[g->nx + 1] = xi[g->nx];
    xhr[g->nx + 1] = xhr[g->nx]; xhi[g->nx + 1] = xhi[g->nx];
    yr[0] = yr[1]; yi[0] = yi[1]; yhr[0] = yhr[1]; yhi[0] = yhi[1];
    yr[g->ny + 1] = yr[g->ny]; yi[g->ny + 1] = yi[g->ny];
    yhr[g->ny + 1] = yhr[g->ny]; yhi[g->ny + 1] = yhi[g->ny];
}

/* The nine stiffness weights of one row (b-values of av_rho/av_mu). */
typedef struct { float pm, mp, pp, mm, p0, m0, zp, zm; } bvals;

/* Mixed-grid FD weights, src/AC/init_A_AC_9p_pml.c:34-40 */
typedef struct { float a, b, c, d, e, idh2; } fdw;

static fdw fd_weights(float dh)
{
    fdw w;
    w.a = 0.6287326; w.b = 0.3712667;
    w.c = 1 - w.a - w.b;
    w.b = 0.25 * w.b; w.c = 0.25 * w.c;
    w.d = 0.4382634; w.e = 1 - w.d;
    w.idh2 = 1.0 / (dh * dh);
    return w;
}

/* One row of the 9-point mixed-grid stencil (init_A_AC_9p_pml.c:68-216,
 * same expressions in init_A_SH_9p_pml.c and init_A_TE_9p_pml.c with unit
 * b-values).  mass[q] = the complex-float mass factor of neighbour q
 * (NW,N,NE,W,C,E,SW,S,SE); coef[q] receives the complex-float coefficient.
 * The TE coefficients are exactly these expressions with all b-values 1:
 * b*d (b = 1.0f) is d exactly, (d + d) equals (2.0*d) exactly. */
static void stencil_row(const fdw *w, const bvals *b, const complex float mass[9],
                        complex float dx0, complex float dy0, complex float dxp,
                        complex float dxm, complex float dyp, complex float dym,
                        complex float coef[9])
{
    const float damp = 0.0;
    const double q = 0.25 * w->idh2;
    complex float t;
    /* NW */
    coef[0] = w->c * mass[0] + w->d * (q * dy0 * b->mm * dym + q * dx0 * b->mm * dxm);
    /* N */
    t = w->b * mass[1]
        + w->d * (q * dy0 * (b->pm * dym + b->mm * dym) + q * dx0 * (-b->pm * dxp - b->mm * dxm))
        + w->e * (dy0 * w->idh2 * b->m0 * dym);
    t += -damp * t;
    coef[1] = t;
    /* NE */
    coef[2] = w->c * mass[2] + w->d * (q * dy0 * b->pm * dym + q * dx0 * b->pm * dxp);
    /* W */
    t = w->b * mass[3]
        + w->d * (q * dy0 * (-b->mp * dyp - b->mm * dym) + q * dx0 * (b->mp * dxm + b->mm * dxm))
        + w->e * (dx0 * w->idh2 * b->m0 * dxm);
    t += -damp * t;
    coef[3] = t;
    /* centre */
    t = w->a * mass[4]
        + w->d * (-0.25 * w->idh2 * dy0 * (b->mp * dyp + b->pm * dym + b->pp * dyp + b->mm * dym)
                  - q * dx0 * (b->mp * dxm + b->pm * dxp + b->pp * dxp + b->mm * dxm))
        + w->e * (-dy0 * w->idh2 * (dyp * b->zp + dym * b->zm) - dx0 * w->idh2 * (dxp * b->p0 + dxm * b->m0));
    t += damp * 4.0 * t;
    coef[4] = t;
    /* E */
    t = w->b * mass[5]
        + w->d * (q * dy0 * (-b->pm * dym - b->pp * dyp) + q * dx0 * (b->pm * dxp + b->pp * dxp))
        + w->e * (dx0 * w->idh2 * b->p0 * dxp);
    t += -damp * t;
    coef[5] = t;
    /* SW */
    coef[6] = w->c * mass[6] + w->d * (q * dy0 * b->mp * dyp + q * dx0 * b->mp * dxm);
    /* S */
    t = w->b * mass[7]
        + w->d * (q * dy0 * (b->mp * dyp + b->pp * dyp) + q * dx0 * (-b->mp * dxm - b->pp * dxp))
        + w->e * (dy0 * w->idh2 * b->zp * dyp);
    t += -damp * t;
    coef[7] = t;
    /* SE */
    coef[8] = w->c * mass[8] + w->d * (q * dy0 * b->pp * dyp + q * dx0 * b->pp * dxp);
}

/* Impedance-matrix assembly as NONZERO triplets in the reference's
 * row-major order with ascending columns:
 *   physics 1 (AC, src/AC/init_A_AC_9p_pml.c:17-220; m0 = vp, m1 = rho),
 *   physics 2 (SH, src/SH/init_A_SH_9p_pml.c:17-222; m0 = vs, m1 = rho),
 *   physics 4 (TE, src/TE/init_A_TE_9p_pml.c:21-243; m0 = epsilon, m1 = sigma).
 * Returns the number of triplets written, or -1 for an unknown physics. */
int port_assemble(const port_grid *g, int physics, float freq, const float *m0, const float *m1,
                  double *ar, double *ai, int *irow, int *icol)
{
    const int nx = g->nx, ny = g->ny;
    const fdw w = fd_weights(g->dh);
    float *pml = malloc(sizeof(float) * 4 * ((nx + 2) + (ny + 2)));
    float *mass_f = NULL, *bh = NULL;
    complex float *mass_c = NULL;
    complex float om2, omega = 0;
    const float mu0 = 4.0 * M_PI * 1e-7;
    int count = 0;
    if (physics != 1 && physics != 2 && physics != 4) { free(pml); return -1; }
    port_pml(g, freq, pml);
    const float *pxr = pml, *pxi = pml + (nx + 2), *pxhr = pml + 2 * (nx + 2), *pxhi = pml + 3 * (nx + 2);
    const float *pyr = pml + 4 * (nx + 2), *pyi = pyr + (ny + 2), *pyhr = pyr + 2 * (ny + 2), *pyhi = pyr + 3 * (ny + 2);

    if (physics == 4) {
        omega = 2.0 * M_PI * (freq + g->s * I);
        om2 = cpowf(2.0 * M_PI * (freq + g->s * I), 2.0);
        mass_c = malloc(sizeof(complex float) * nx * ny);
        for (int k = 0; k < nx * ny; k++) {
            complex float epse = m0[k] + (m1[k] / omega) * I;   /* init_A_TE_9p_pml.c:76 */
            mass_c[k] = om2 * mu0 * epse;
        }
    } else {
        om2 = (physics == 1) ? cpowf(2.0 * M_PI * (freq - g->s * I), 2.0)
                             : cpowf(2.0 * M_PI * (freq + g->s * I), 2.0);
        mass_f = malloc(sizeof(float) * nx * ny);
        /* halo-padded stiffness field: b = 1/rho (init_mat_AC.c:18-37) or
         * mu = rho*vs^2 (init_mat_SH.c:18-31), (ny+2) x (nx+2) */
        bh = malloc(sizeof(float) * (nx + 2) * (ny + 2));
        for (int j = 1; j <= ny; j++)
            for (int i = 1; i <= nx; i++) {
                int k = (j - 1) * nx + (i - 1);
                if (physics == 1) {
                    mass_f[k] = 1.0 / (m1[k] * m0[k] * m0[k]);
                    bh[j * (nx + 2) + i] = 1.0 / m1[k];
                } else {
                    mass_f[k] = m1[k];
                    bh[j * (nx + 2) + i] = m1[k] * m0[k] * m0[k];
                }
            }
        for (int j = 1; j <= ny; j++) { bh[j * (nx + 2)] = bh[j * (nx + 2) + 1]; bh[j * (nx + 2) + nx + 1] = bh[j * (nx + 2) + nx]; }
        for (int i = 0; i <= nx + 1; i++) { bh[i] = bh[(nx + 2) + i]; bh[(ny + 1) * (nx + 2) + i] = bh[ny * (nx + 2) + i]; }
    }

    for (int j = 1; j <= ny; j++) {
        for (int i = 1; i <= nx; i++) {
            const int k = (j - 1) * nx + (i - 1);
            bvals b;
            if (physics == 1) {           /* pointwise buoyancy, src/av_rho.c:32-48 */
                float v = bh[j * (nx + 2) + i];
                b.pm = b.mp = b.pp = b.mm = b.p0 = b.m0 = b.zp = b.zm = v;
            } else if (physics == 2) {    /* averaged modulus, src/SH/av_mu.c:12-28 */
#define MU(jj, ii) bh[(jj) * (nx + 2) + (ii)]
                b.pm = 0.25 * (MU(j, i) + MU(j, i + 1) + MU(j - 1, i) + MU(j - 1, i + 1));
                b.mp = 0.25 * (MU(j, i) + MU(j, i - 1) + MU(j + 1, i) + MU(j + 1, i - 1));
                b.pp = 0.25 * (MU(j, i) + MU(j, i + 1) + MU(j + 1, i) + MU(j + 1, i + 1));
                b.mm = 0.25 * (MU(j, i) + MU(j, i - 1) + MU(j - 1, i) + MU(j - 1, i - 1));
                b.p0 = 0.5 * (MU(j, i) + MU(j, i + 1));
                b.m0 = 0.5 * (MU(j, i) + MU(j, i - 1));
                b.zp = 0.5 * (MU(j, i) + MU(j + 1, i));
                b.zm = 0.5 * (MU(j, i) + MU(j - 1, i));
#undef MU
            } else {
                b.pm = b.mp = b.pp = b.mm = b.p0 = b.m0 = b.zp = b.zm = 1.0f;
            }
            complex float mass[9];
            for (int q = 0; q < 9; q++) {
                int di = q % 3 - 1, dj = q / 3 - 1;
                int ii = i + di, jj = j + dj;
                if (ii < 1 || ii > nx || jj < 1 || jj > ny) { mass[q] = 0; continue; }
                int kk = (jj - 1) * nx + (ii - 1);
                mass[q] = (physics == 4) ? mass_c[kk] : om2 * mass_f[kk];
            }
            complex float dy0 = pyr[j] + pyi[j] * I, dx0 = pxr[i] + pxi[i] * I;
            complex float dyp = pyhr[j] + pyhi[j] * I, dym = pyhr[j - 1] + pyhi[j - 1] * I;
            complex float dxp = pxhr[i] + pxhi[i] * I, dxm = pxhr[i - 1] + pxhi[i - 1] * I;
            complex float coef[9];
            stencil_row(&w, &b, mass, dx0, dy0, dxp, dxm, dyp, dym, coef);
            for (int q = 0; q < 9; q++) {
                int di = q % 3 - 1, dj = q / 3 - 1;
                int ii = i + di, jj = j + dj;
                if (ii < 1 || ii > nx || jj < 1 || jj > ny) continue;
                ar[count] = crealf(coef[q]);
                ai[count] = cimagf(coef[q]);
                irow[count] = k;
                icol[count] = k + di + dj * nx;
                count++;
            }
        }
    }
    free(pml); free(mass_f); free(mass_c); free(bh);
    return count;
}

/* Spike source vector, src/AC/RHS_source_AC.c:11-58 (amp 1) and
 * src/TE/RHS_source_TE.c:11-61 (amp -i*Omega*mu0).  rhs is NX*NY long. */
void port_rhs_source(const port_grid *g, int physics, float freq, float xsrc, float ysrc,
                     double *rr, double *ri)
{
    float amp_r = 1.0f, amp_i = 0.0f;
    int nxs = iround_f(xsrc / g->dh) + g->npml;
    int nys = iround_f(ysrc / g->dh) + g->fsshift;
    int ks = nxs + (nys - 1) * g->nx;
    if (physics == 4) {
        complex float om = 2.0 * M_PI * (freq + g->s * I);
        float mu0 = 4.0 * M_PI * 1e-7;
        amp_r = -creal((om * mu0 * I) * (1.0 + 0.0 * I));
        amp_i = -cimag((om * mu0 * I) * (1.0 + 0.0 * I));
    }
    memset(rr, 0, sizeof(double) * g->nx * g->ny);
    memset(ri, 0, sizeof(double) * g->nx * g->ny);
    rr[ks] = amp_r / (g->dh * g->dh);
    ri[ks] = amp_i / (g->dh * g->dh);
}

/* Solution vector -> float wavefield with the reference's one-slot shift,
 * src/vec2mat.c:19-26: field[k] = (float) x[k+1]; x must have NX*NY+1
 * entries (the last one is defined as 0). */
void port_vec2mat(int nxny, const double *xr, const double *xi, float *pr, float *pi)
{
    for (int k = 0; k < nxny; k++) { pr[k] = (float)xr[k + 1]; pi[k] = (float)xi[k + 1]; }
}

/* Receiver gather, src/AC/calc_seis_AC.c:18-22; ishot and nfreq 1-based,
 * output index (0-based) = t + ntr*(ishot-1) + ntr*nshots*(nfreq-1). */
void port_calc_seis(const port_grid *g, const float *pr, const float *pi, int ntr, const int *recx,
                    const int *recy, int ishot, int nshots, int nfreq, float *sr, float *si)
{
    for (int t = 0; t < ntr; t++) {
        int o = t + ntr * (ishot - 1) + ntr * nshots * (nfreq - 1);
        int k = (recy[t] + g->fsshift - 1) * g->nx + (recx[t] + g->npml - 1);
        sr[o] = pr[k]; si[o] = pi[k];
    }
}

/* Residuals and misfit of one shot, src/AC/calc_res_AC.c:10-95.  obs/cal
 * point at this shot's ntr samples.  The local misfit starts at 0 (the
 * reference leaves it uninitialised when stf_inv == 0). */
float port_calc_res(const float *calr, const float *cali, const float *obsr, const float *obsi,
                    int ntr, int stf_inv, int invmat, int misfit, float *resr, float *resi, float *stf)
{
    float l2 = 0.0f;
    complex float wien = 1.0f, res = 0.0f;
    if (stf_inv == 1) {
        complex float num = 0.0 + 0.0 * I, den = 0.0 + 0.0 * I;
        for (int t = 0; t < ntr; t++) {
            num += conj(calr[t] + cali[t] * I) * (obsr[t] + obsi[t] * I);
            den += conj(obsr[t] + obsi[t] * I) * (obsr[t] + obsi[t] * I);
        }
        wien = num / den;
    }
    if (stf_inv == 0) wien = 1.0 + 0.0 * I;
    stf[0] = crealf(wien); stf[1] = cimagf(wien);
    for (int t = 0; t < ntr; t++) {
        if (invmat == 1) {
            if (misfit == 1) res = ((obsr[t] + obsi[t] * I) - (wien * (calr[t] + cali[t] * I))) / cabsf(wien);
            if (misfit == 2) res = clogf(obsr[t] + obsi[t] * I) - clogf(calr[t] + cali[t] * I);
            if (misfit == 3) res = cargf(calr[t] + cali[t] * I) - cargf(obsr[t] + obsi[t] * I);
        }
        if (invmat == 2) res = obsr[t] + obsi[t] * I;
        resr[t] = crealf(res); resi[t] = cimagf(res);
        if ((obsr[t] < 1e-20) && (obsi[t] < 1e-20)) { resr[t] = 0.0f; resi[t] = 0.0f; }
        l2 += creal(res * conj(res));
    }
    return l2;
}

/* Adjoint source, src/AC/RHS_source_AC_adj.c:17-34: conj(res)/DH^2 at the
 * receivers (later receivers overwrite earlier ones on the same point). */
void port_rhs_adj(const port_grid *g, const float *resr, const float *resi, int ntr,
                  const int *recx, const int *recy, double *rr, double *ri)
{
    memset(rr, 0, sizeof(double) * g->nx * g->ny);
    memset(ri, 0, sizeof(double) * g->nx * g->ny);
    for (int t = 0; t < ntr; t++) {
        int k = (recx[t] + g->npml) + (recy[t] + g->fsshift - 1) * g->nx;
        rr[k] = resr[t] / (g->dh * g->dh);
        ri[k] = -resi[t] / (g->dh * g->dh);
    }
}

/* One shot's AC gradient accumulated into grad, src/AC/ass_grad_AC.c:22-52
 * (no per-shot taper). */
void port_ass_grad_ac(const port_grid *g, float freq, const float *stf, const float *fr,
                      const float *fi, const float *lr, const float *li, const float *vp,
                      const float *rho, float *grad)
{
    complex float wien = stf[0] + stf[1] * I;
    complex float om2 = cpowf(((2.0 * M_PI * freq) - (I * g->s)), 2.0);
    for (int k = 0; k < g->nx * g->ny; k++) {
        float gs = -2.0 * creal(om2 * (wien / cabsf(wien)) * (fr[k] + fi[k] * I)
                               * (1.0 / (rho[k] * vp[k] * vp[k] * vp[k])) * (lr[k] + li[k] * I));
        grad[k] += gs;
    }
}

/* One shot's TE gradients, src/TE/ass_grad_TE.c:22-59. */
void port_ass_grad_te(const port_grid *g, float freq, const float *stf, const float *fr,
                      const float *fi, const float *lr, const float *li, float *gsig, float *geps)
{
    complex float wien = stf[0] + stf[1] * I;
    complex float om = 2.0 * M_PI * (freq + (I * g->s));
    complex float om2 = cpowf(2.0 * M_PI * (freq + (I * g->s)), 2.0);
    for (int k = 0; k < g->nx * g->ny; k++) {
        float a = creal((wien / cabsf(wien)) * (fr[k] + fi[k] * I) * (om * I) * (lr[k] + li[k] * I));
        float b = creal(om2 * (wien / cabsf(wien)) * (fr[k] + fi[k] * I) * (lr[k] + li[k] * I));
        gsig[k] += a;
        geps[k] += b;
    }
}

/* PML taper coefficients of cp_grad_frame (PML_grad == 3),
 * src/cp_grad_frame.c:108-170: returns the [NY][NX] multiplier field. */
void port_grad_frame_coeff(const port_grid *g, float *coef)
{
    const int nx = g->nx, ny = g->ny, npml = g->npml;
    float *c = malloc(sizeof(float) * (npml + 1));
    float damping = 60.0, amp = 1.0 - damping / 100.0;
    float a = sqrt(-log(amp) / ((npml - 1) * (npml - 1)));
    for (int p = 1; p <= npml; p++) c[p] = exp(-(a * a * (npml - p) * (npml - p)));
    for (int k = 0; k < nx * ny; k++) coef[k] = 1.0f;
#define C(jj, ii) coef[((jj) - 1) * nx + (ii) - 1]
    for (int p = 1; p <= npml; p++)
        for (int j = p; j <= ny - p + 1; j++) C(j, p) = c[p];
    for (int p = 1; p <= npml; p++)
        for (int j = p; j <= ny - p + 1; j++) C(j, nx - p + 1) = c[p];
    if (g->free_surf == 0)
        for (int p = 1; p <= npml; p++)
            for (int i = p; i <= nx - p + 1; i++) C(p, i) = c[p];
    for (int p = 1; p <= npml; p++)
        for (int i = p; i <= nx - p + 1; i++) C(ny - p + 1, i) = c[p];
#undef C
    free(c);
}

/* Apply the frame taper in the reference's region order (left, right, top,
 * bottom; corners are multiplied once per region that covers them),
 * src/cp_grad_frame.c:172-214.  NaN repair is not restated. */
void port_cp_grad_frame(const port_grid *g, float *grad)
{
    const int nx = g->nx, ny = g->ny, npml = g->npml;
    const int nx0 = nx - 2 * npml, ny0 = ny - npml - g->fsshift;
    float *coef = malloc(sizeof(float) * nx * ny);
    port_grad_frame_coeff(g, coef);
#define G(jj, ii) grad[((jj) - 1) * nx + (ii) - 1]
#define C(jj, ii) coef[((jj) - 1) * nx + (ii) - 1]
    for (int i = 1; i <= npml; i++) for (int j = 1; j <= ny; j++) G(j, i) *= C(j, i);
    for (int i = npml + nx0 + 1; i <= nx; i++) for (int j = 1; j <= ny; j++) G(j, i) *= C(j, i);
    if (g->free_surf == 0)
        for (int i = 1; i <= nx; i++) for (int j = 1; j <= npml; j++) G(j, i) *= C(j, i);
    for (int i = 1; i <= nx; i++) for (int j = g->fsshift + ny0 + 1; j <= ny; j++) G(j, i) *= C(j, i);
#undef G
#undef C
    free(coef);
}

/* Gradient scalars: AC Omega^2 = cpowf((2 pi f) - iS, 2) (ass_grad_AC.c:22);
 * TE Omega = 2 pi (f + iS), Omega^2 = cpowf(2 pi (f + iS), 2) (ass_grad_TE.c:22-23). */
void port_gradient_scalars(const port_grid *g, int physics, float freq, float *om2, float *om)
{
    complex float o2, o = 0.0f;
    if (physics == 4) {
        o = 2.0 * M_PI * (freq + (I * g->s));
        o2 = cpowf(2.0 * M_PI * (freq + (I * g->s)), 2.0);
    } else {
        o2 = cpowf(((2.0 * M_PI * freq) - (I * g->s)), 2.0);
    }
    om2[0] = crealf(o2); om2[1] = cimagf(o2);
    om[0] = crealf(o); om[1] = cimagf(o);
}

/* Gaussian smoothing of the gradient, src/gauss_filt.c:10-141 (SPATFILTER=1
 * in precond(), src/precond.c:18).  grad [NY][NX] is filtered in place;
 * window and weights in the reference's float / double arithmetic, edges
 * extended by their last value (gauss_filt.c:72-100), float accumulation
 * with taps along x outer and along y inner. */
void port_gauss_filt(const port_grid *g, float vref, float fc_low, float fsg, float fsg1, float *grad)
{
    const int nx = g->nx, ny = g->ny;
    const float lam = vref / fc_low;
    int fx = round((fsg * lam) / g->dh), fy = round((fsg1 * lam) / g->dh);
    int hx, hy, ii, jj, i, j, nwx;
    float sgx, sgy, sx, sy, total = 0.0, *wt, *src;
    if (fx == 0 || fy == 0) return;
    if (fx % 2 == 0) fx += (fx > 0) ? 1 : -1;
    if (fy % 2 == 0) fy += (fy > 0) ? 1 : -1;
    hx = abs(fx) / 2; hy = abs(fy) / 2;
    sgx = hx / 2; sgy = hy / 2;
    sx = 2.0 * sgx * sgx; sy = 2.0 * sgy * sgy;
    nwx = 2 * hx + 1;
    wt = malloc(sizeof(float) * (size_t)nwx * (2 * hy + 1));
    src = malloc(sizeof(float) * (size_t)nx * ny);
    for (ii = -hx; ii <= hx; ii++)
        for (jj = -hy; jj <= hy; jj++) {
            float v = exp(-((ii * ii) / sx) - ((jj * jj) / sy));
            wt[(jj + hy) * nwx + ii + hx] = v;
            total += v;
        }
    /* gauss_filt.c:114-120 normalises over i <= filt_size_x, j <= filt_size_y:
     * with a negative size the loop is empty and the weights stay raw */
    if (fx > 0 && fy > 0)
        for (i = 0; i < nwx * (2 * hy + 1); i++) wt[i] /= total;
    memcpy(src, grad, sizeof(float) * (size_t)nx * ny);
    for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
            float acc = 0.0;
            for (ii = -hx; ii <= hx; ii++) {
                int x = i + ii;
                x = x < 0 ? 0 : (x >= nx ? nx - 1 : x);
                for (jj = -hy; jj <= hy; jj++) {
                    int y = j + jj;
                    y = y < 0 ? 0 : (y >= ny ? ny - 1 : y);
                    acc += src[y * nx + x] * wt[(jj + hy) * nwx + ii + hx];
                }
            }
            grad[j * nx + i] = acc;
        }
    free(wt);
    free(src);
}

/* apply_hess_AC, src/AC/apply_hess_AC.c:11-40: MAX_HESS is the largest
 * fabs(hess) (a float; entries whose fabs is not > the running maximum, NaN
 * included, are skipped), then grad *= 1.0 / (hess + EPS_HESS * MAX_HESS):
 * the denominator in float, the reciprocal and the product in double, the
 * result stored as float.  Returns MAX_HESS. */
float port_apply_hess(int n, float eps_hess, float *grad, const float *hess)
{
    float max_hess = 0.0f;
    int k;
    for (k = 0; k < n; k++)
        if (fabs(hess[k]) > max_hess) max_hess = fabs(hess[k]);
    for (k = 0; k < n; k++) {
        const float den = hess[k] + eps_hess * max_hess;
        const double q = 1.0 / den;
        grad[k] = (float)(grad[k] * q);
    }
    return max_hess;
}

/* ---- l-BFGS (src/LBFGS.c:12-250 for one parameter class, src/TE/LBFGS_TE.c
 * for two) on flat arrays.  Vectors of length nvec = nclass * NX * NY are in
 * the reference's order: class outer, then x (i) outer, y (j) inner, 0-based;
 * y, s hold m such vectors (slot k at offset (k-1) * nvec).  grad, gradm,
 * model, hess and hgrad are [nclass][NY][NX] row-major.  old_grad /
 * old_model hold what the reference's "<JACOBIAN>_p.old" / "_p_vp.old"
 * files hold (grad and model of the previous call) in vector order and are
 * overwritten with this call's.  hess == NULL: initial Hessian gamma
 * (LBFGS.c:124-126, LBFGS_TE.c HESSIAN = 0); else q / (hess + eps *
 * MAX_HESS) per class (LBFGS_TE.c HESSIAN != 0).  first != 0: Hgrad =
 * gradm (iter == 1 / LBFGS_RESET == 1).  Float arithmetic and summation
 * order as the reference (dotp, src/dotp.c:10-35, sums in float). */
static float port_dotp(const float *v1, const float *v2, int n)
{
    float tmp = 0.0f;
    for (int i = 0; i < n; i++) tmp += v1[i] * v2[i];
    return tmp;
}

void port_lbfgs(const port_grid *g, int nclass, int m, int pointer, int first, float *y, float *s,
                const float *grad, const float *gradm, const float *model, const float *hess, float eps_hess,
                float *old_grad, float *old_model, float *q, float *r, float *scal, float *hgrad)
{
    const int nx = g->nx, ny = g->ny, n = nx * ny, nvec = nclass * n;
    float *rho = scal, *alpha = scal + m;   /* scal: 2 m + 1 floats, the last = gamma */
    int c, i, j, k, h;
    if (!first) {
        h = nvec * (pointer - 1);
        for (c = 0; c < nclass; c++)
            for (i = 0; i < nx; i++)
                for (j = 0; j < ny; j++, h++) {
                    const int gi = c * n + j * nx + i, v = h - nvec * (pointer - 1);
                    y[h] = grad[gi] - old_grad[v];
                    s[h] = model[gi] - old_model[v];
                }
        {
            const float *yp = y + nvec * (pointer - 1), *sp = s + nvec * (pointer - 1);
            const float nom = port_dotp(yp, sp, nvec), den = port_dotp(yp, yp, nvec);
            scal[2 * m] = nom / den;
        }
        for (k = 1; k <= m; k++) {
            const float sum = port_dotp(y + nvec * (k - 1), s + nvec * (k - 1), nvec);
            rho[k - 1] = (fabs(sum) > 0.0) ? 1.0 / sum : 0.0;
        }
        h = 0;
        for (c = 0; c < nclass; c++)
            for (i = 0; i < nx; i++)
                for (j = 0; j < ny; j++) q[h++] = gradm[c * n + j * nx + i];
        for (k = m; k >= 1; k--) {
            const float sum = port_dotp(s + nvec * (k - 1), q, nvec);
            alpha[k - 1] = rho[k - 1] * sum;
            for (i = 0; i < nvec; i++) q[i] = q[i] - alpha[k - 1] * y[nvec * (k - 1) + i];
        }
        if (!hess) {
            for (i = 0; i < nvec; i++) r[i] = scal[2 * m] * q[i];
        } else {
            h = 0;
            for (c = 0; c < nclass; c++) {
                float mx = 0.0f;
                for (k = 0; k < n; k++)
                    if (fabs(hess[c * n + k]) > mx) mx = fabs(hess[c * n + k]);
                for (i = 0; i < nx; i++)
                    for (j = 0; j < ny; j++, h++) r[h] = q[h] / (hess[c * n + j * nx + i] + eps_hess * mx);
            }
        }
        for (k = 1; k <= m; k++) {
            const float sum = port_dotp(y + nvec * (k - 1), r, nvec);
            const float beta = rho[k - 1] * sum;
            for (i = 0; i < nvec; i++) r[i] = r[i] + s[nvec * (k - 1) + i] * (alpha[k - 1] - beta);
        }
        h = 0;
        for (c = 0; c < nclass; c++)
            for (i = 0; i < nx; i++)
                for (j = 0; j < ny; j++) hgrad[c * n + j * nx + i] = r[h++];
    } else {
        for (k = 0; k < nvec; k++) hgrad[k] = gradm[k];
    }
    for (c = 0; c < nclass; c++) port_cp_grad_frame(g, hgrad + c * n);
    h = 0;
    for (c = 0; c < nclass; c++)
        for (i = 0; i < nx; i++)
            for (j = 0; j < ny; j++, h++) {
                old_grad[h] = grad[c * n + j * nx + i];
                old_model[h] = model[c * n + j * nx + i];
            }
}

/* rot_LBFGS_vec, src/rot_LBFGS_vec.c:10-24: slots 2..m move to 1..m-1 */
void port_lbfgs_rotate(int m, int nvec, float *y, float *s)
{
    for (int k = 0; k < (m - 1) * nvec; k++) {
        y[k] = y[k + nvec];
        s[k] = s[k + nvec];
    }
}

/* check_descent (src/check_descent.c:17-19) / check_descent_multi_para_TE
 * (src/TE/check_descent_multi_para_TE.c:21-26): p = -nom / denom from
 * per-class dotp_matrix sums (x outer, y inner) added in float.  Grids are
 * [nclass][NY][NX] row-major. */
float port_check_descent(const port_grid *g, int nclass, const float *hgrad, const float *grad)
{
    const int nx = g->nx, ny = g->ny, n = nx * ny;
    float nom = 0.0f, den = 0.0f;
    for (int c = 0; c < nclass; c++) {
        float a = 0.0f, b = 0.0f;
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) {
                const int k = c * n + j * nx + i;
                a += hgrad[k] * grad[k];
                b += grad[k] * grad[k];
            }
        if (c == 0) { nom = a; den = b; }
        else { nom += a; den += b; }
    }
    return -nom / den;
}

/* precond (src/precond.c:10-24) without its gauss_filt step (restated in
 * port_gauss_filt): taper_grad_hor (src/taper_grad_hor.c:20-31) when
 * taper_hor, then taper_grad_file (src/taper_grad_file.c:18-70) when taper
 * (NX0 x NY0 floats, x outer) is given.  grad [NY][NX] in place. */
void port_precond_tapers(const port_grid *g, int taper_hor, int gradt2, const float *taper, float *grad)
{
    const int nx = g->nx, ny = g->ny, npml = g->npml, fs = g->fsshift;
    const int nx0 = nx - 2 * npml, ny0 = ny - npml - fs;
    int i, j;
#define G(jj, ii) grad[((jj) - 1) * nx + (ii) - 1]
    if (taper_hor)
        for (j = 1; j <= ny; j++)
            for (i = 1; i <= nx; i++)
                if (j <= gradt2 + fs) G(j, i) = 0.0f;
    if (taper) {
        int t = 0;
        for (i = 1; i <= nx0; i++)
            for (j = 1; j <= ny0; j++) G(j + fs, i + npml) *= taper[t++];
        for (i = 1; i <= npml; i++)
            for (j = 1; j <= ny; j++) G(j, i) = G(j, npml + 1);
        for (i = npml + nx0 + 1; i <= nx; i++)
            for (j = 1; j <= ny; j++) G(j, i) = G(j, npml + nx0);
        if (g->free_surf == 1)
            for (i = 1; i <= nx; i++)
                for (j = 1; j <= npml; j++) G(j, i) = G(npml + 1, i);
        for (i = 1; i <= nx; i++)
            for (j = fs + ny0 + 1; j <= ny; j++) G(j, i) = G(fs + ny0, i);
    }
#undef G
}

/* Radial taper field of one centre (xc, yc) in metres, as taper_grad_shot
 * evaluates it for the shot's source (src/taper_grad_shot.c:33-37, 47-56)
 * and for each receiver with centre recpos * DH (:66-76):
 * coef = f0 + (1 - f0) (1/2 - 1/2 cos(pi r / R))^a for r <= R, 1 beyond,
 * x = i DH and y = j DH over the whole grid (no PML shift). */
void port_srt_field(const port_grid *g, float xc, float yc, float radius, float *coef)
{
    float frh = 0.1, f0 = 1e-3;
    float a = -(log(frh - f0) - log(1.0 - f0)) / log(2.0);
    for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++) {
            float x = i * g->dh, y = j * g->dh;
            float r = sqrt(pow((x - xc), 2.0) + pow((y - yc), 2.0));
            float t = 1.0;
            if (r <= radius) t = f0 + (1.0 - f0) * pow((0.5 - 0.5 * cos(M_PI * r / radius)), a);
            coef[(j - 1) * g->nx + i - 1] = t;
        }
}

/* taper_grad_shot1 (src/taper_grad_shot1.c:25-57): 1e-5 on the
 * (2 F + 1)^2 squares around every source (centre iround(x / DH)) and every
 * receiver (its grid indices); points off the grid are skipped. */
void port_taper_grad_shot1(const port_grid *g, int filtsize, int nshots, const float *sx, const float *sy, int ntr,
                           const int *rx, const int *ry, float *grad)
{
    for (int n = 0; n < nshots + ntr; n++) {
        const int i1 = n < nshots ? iround_f(sx[n] / g->dh) : rx[n - nshots];
        const int j1 = n < nshots ? iround_f(sy[n] / g->dh) : ry[n - nshots];
        for (int i = i1 - filtsize; i <= i1 + filtsize; i++)
            for (int j = j1 - filtsize; j <= j1 + filtsize; j++)
                if (i >= 1 && i <= g->nx && j >= 1 && j <= g->ny) grad[(j - 1) * g->nx + i - 1] = 1e-5f;
    }
}
