/*
 * Host-side per-frequency set-up scalars and 1-D profiles of the engine.
 *
 * These are O(1) or O(NX+NY) per frequency, computed on the host exactly as
 * the reference computes them (same C99 complex types, gcc, no FMA) and
 * uploaded to the device; all O(NX*NY) work runs in the CUDA kernels.  The
 * file is C, not C++, because the roundings of C99 complex float/double
 * arithmetic (complex float division, promotion of complex float to complex
 * double next to a double literal, glibc cpowf) are part of the reference's
 * numerics that the assembly kernel must reproduce bit for bit.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "host_setup.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* mixed-grid weights a, b, c, d, e and 1/DH^2: src/AC/init_A_AC_9p_pml.c:34-43 */
void gmh_fd_weights(float dh, float w[6])
{
    float a = 0.6287326, b = 0.3712667, c, d, e, idh2;
    c = 1 - a - b;
    b = 0.25 * b;
    c = 0.25 * c;
    d = 0.4382634;
    e = 1 - d;
    idh2 = 1.0 / (dh * dh);
    w[0] = a; w[1] = b; w[2] = c; w[3] = d; w[4] = e; w[5] = idh2;
}

/* 1-D PML stretch profiles, src/pml_pro.c:20-160.  out holds 4 x-arrays of
 * NX+2 (node r/i, half-node r/i) followed by 4 y-arrays of NY+2. */
void gmh_pml(int nx, int ny, float dh, int npml, int free_surf, float a0_pml, float s,
             float freq, float *out)
{
    const int nxa = nx + 2, nya = ny + 2;
    float *xr = out, *xi = out + nxa, *xhr = out + 2 * nxa, *xhi = out + 3 * nxa;
    float *yr = out + 4 * nxa, *yi = yr + nya, *yhr = yi + nya, *yhi = yhr + nya;
    const float half_pi = M_PI / 2.0;
    const complex float ci = 0.0 + 1.0 * I;
    const float width = npml * dh;
    const complex float omega = 2.0 * M_PI * (freq - I * s);
    int k;
    for (k = 0; k < nxa; k++) { xr[k] = 1.0f; xi[k] = 0.0f; xhr[k] = 1.0f; xhi[k] = 0.0f; }
    for (k = 0; k < nya; k++) { yr[k] = 1.0f; yi[k] = 0.0f; yhr[k] = 1.0f; yhi[k] = 0.0f; }
    for (k = 1; k <= npml; k++) {
        const float x = k * dh;
        const float xh = x + 0.5 * dh;
        const float damp = a0_pml * (1.0 - cos((width - x) * half_pi / width));
        const float damph = a0_pml * (1.0 - cos((width - xh) * half_pi / width));
        const complex double node = 1.0 / (1.0 + damp / (ci * omega));
        const complex double half = 1.0 / (1.0 + damph / (ci * omega));
        xr[k] = creal(node); xi[k] = cimag(node);
        xhr[k] = creal(half); xhi[k] = cimag(half);
        yr[k] = xr[k]; yi[k] = xi[k]; yhr[k] = xhr[k]; yhi[k] = xhi[k];
        xr[nx - k + 1] = xr[k]; xi[nx - k + 1] = xi[k];
        xhr[nx - k + 1] = xhr[k]; xhi[nx - k + 1] = xhi[k];
        yr[ny - k + 1] = xr[k]; yi[ny - k + 1] = xi[k];
        yhr[ny - k + 1] = xhr[k]; yhi[ny - k + 1] = xhi[k];
        if (free_surf == 1) { yr[k] = 1.0f; yi[k] = 0.0f; yhr[k] = 1.0f; yhi[k] = 0.0f; }
    }
    xr[0] = xr[1]; xi[0] = xi[1]; xhr[0] = xhr[1]; xhi[0] = xhi[1];
    xr[nx + 1] = xr[nx]; xi[nx + 1] = xi[nx]; xhr[nx + 1] = xhr[nx]; xhi[nx + 1] = xhi[nx];
    yr[0] = yr[1]; yi[0] = yi[1]; yhr[0] = yhr[1]; yhi[0] = yhi[1];
    yr[ny + 1] = yr[ny]; yi[ny + 1] = yi[ny]; yhr[ny + 1] = yhr[ny]; yhi[ny + 1] = yhi[ny];
}

/* Per-frequency scalars of the assembly:
 *   om2    = Omega^2 via glibc cpowf, AC: (2 pi (f - iS))^2
 *            (init_A_AC_9p_pml.c:50), SH/TE: (2 pi (f + iS))^2
 *            (init_A_SH_9p_pml.c:50, init_A_TE_9p_pml.c:55);
 *   om     = TE Omega = 2 pi (f + iS) (init_A_TE_9p_pml.c:54);
 *   om2mu0 = TE Omega^2 * mu0, mu0 = 4 pi 1e-7 (init_A_TE_9p_pml.c:58). */
void gmh_assembly_scalars(int physics, float freq, float s, float om2[2], float om[2], float om2mu0[2])
{
    complex float o2, o = 0.0f, o2m;
    const float mu0 = 4.0 * M_PI * 1e-7;
    if (physics == 1) {
        o2 = cpowf(2.0 * M_PI * (freq - s * I), 2.0);
    } else {
        o2 = cpowf(2.0 * M_PI * (freq + s * I), 2.0);
        o = 2.0 * M_PI * (freq + s * I);
    }
    o2m = o2 * mu0;
    om2[0] = crealf(o2); om2[1] = cimagf(o2);
    om[0] = crealf(o); om[1] = cimagf(o);
    om2mu0[0] = crealf(o2m); om2mu0[1] = cimagf(o2m);
}

/* Spike-source amplitude over DH^2 as stored into the double RHS:
 * AC/SH src/AC/RHS_source_AC.c:48-53 (amp 1), TE src/TE/RHS_source_TE.c:40-55
 * (amp = -i Omega mu0). */
void gmh_source_amp(int physics, float freq, float s, float dh, double amp[2])
{
    float ar = 1.0f, ai = 0.0f;
    if (physics == 4) {
        const complex float omega = 2.0 * M_PI * (freq + s * I);
        const float mu0 = 4.0 * M_PI * 1e-7;
        ar = -creal((omega * mu0 * I) * (1.0 + 0.0 * I));
        ai = -cimag((omega * mu0 * I) * (1.0 + 0.0 * I));
    }
    amp[0] = ar / (dh * dh);
    amp[1] = ai / (dh * dh);
}

/* Spike amplitude of an external source wavelet (READ_WAVELET = 1): the
 * float amplitude read_stf_dft returns, over DH^2 in float as RHS_source_AC
 * / RHS_source_TE divide it (src/AC/RHS_source_AC.c:40-55). */
void gmh_wavelet_amp(const float a[2], float dh, double amp[2])
{
    amp[0] = a[0] / (dh * dh);
    amp[1] = a[1] / (dh * dh);
}

/* The DFT of read_stf_dft (src/read_stf_dft.c:24-71) at one frequency, in
 * its float / double evaluation order: t = (j - 1) dt in float, each term
 * w_j cos(2 t f pi) dt in double added to the float sum.  The reference
 * copies the trace samples one place down (wavelet[j] = data[j] for
 * j = 1 .. ns, from data[0 .. ns - 1] read), so the DFT uses samples 1 ..
 * ns - 1 of the file, at times 0 .. (ns - 2) dt, and a last sample read
 * from beyond the ones in the file; that sample is taken as 0 here.
 * dt = sample interval [mus] / 1e6 (PHYSICS <= 3) or [ns] / 1e12 (TE). */
void gmh_stf_dft(const float *samples, int ns, int ndt, int physics, float freq, float amp[2])
{
    float dt, t, w;
    int j;
    if (physics <= 3) dt = ndt / 1e6;
    else dt = ndt / 1e12;
    amp[0] = 0.0;
    amp[1] = 0.0;
    for (j = 1; j <= ns; j++) {
        w = j < ns ? samples[j] : 0.0f;
        t = (j - 1) * dt;
        amp[0] += w * cos(2.0 * t * freq * M_PI) * dt;
        amp[1] += w * sin(2.0 * t * freq * M_PI) * dt;
    }
}

/* Amplitude of the receiver spike of the Hessian's Green's functions:
 * AC amp/(DH*DH) with float amp = 1 (src/AC/RHS_source_AC_hess.c:26-33, a
 * float quotient); TE 1.0/(DH*DH) (src/TE/RHS_source_TE_hess.c:38, a double
 * quotient). */
double gmh_hess_green_amp(int physics, float dh)
{
    if (physics == 4) return 1.0 / (dh * dh);
    const float amp = 1.0f;
    return amp / (dh * dh);
}

/* Gradient scalars: AC Omega^2 = cpowf((2 pi f) - iS, 2) (ass_grad_AC.c:22);
 * TE Omega = 2 pi (f + iS), Omega^2 = cpowf(2 pi (f + iS), 2)
 * (ass_grad_TE.c:22-23). */
void gmh_gradient_scalars(int physics, float freq, float s, float om2[2], float om[2])
{
    complex float o2, o = 0.0f;
    if (physics == 4) {
        o = 2.0 * M_PI * (freq + (I * s));
        o2 = cpowf(2.0 * M_PI * (freq + (I * s)), 2.0);
    } else {
        o2 = cpowf(((2.0 * M_PI * freq) - (I * s)), 2.0);
    }
    om2[0] = crealf(o2); om2[1] = cimagf(o2);
    om[0] = crealf(o); om[1] = cimagf(o);
}

/* |w| and w/|w| of the source-wavelet estimate, as ass_grad_AC forms
 * (wien/cabsf(wien)) (src/AC/ass_grad_AC.c:30). */
void gmh_stf_unit(const float stf[2], float unit[2])
{
    const complex float w = stf[0] + stf[1] * I;
    const complex float u = w / cabsf(w);
    unit[0] = crealf(u); unit[1] = cimagf(u);
}

/* Wiener source estimate from accumulated sums, src/AC/calc_res_AC.c:40:
 * wien = num / den in complex float. */
void gmh_wiener(const float num[2], const float den[2], float wien[2])
{
    const complex float a = num[0] + num[1] * I, b = den[0] + den[1] * I;
    const complex float w = a / b;
    wien[0] = crealf(w); wien[1] = cimagf(w);
}

/* PML taper of cp_grad_frame (PML_grad = 3), src/cp_grad_frame.c:108-170:
 * coefficient field [NY][NX] and per-point multiplicity (how many of the
 * reference's left/right/top/bottom passes multiply the point). */
void gmh_grad_frame(int nx, int ny, int npml, int free_surf, float *coef, unsigned char *passes)
{
    const int fsshift = free_surf ? 0 : npml;
    const int nx0 = nx - 2 * npml, ny0 = ny - npml - fsshift;
    float c[1024];
    float damping = 60.0, amp = 1.0 - damping / 100.0, a;
    int p, i, j;
    if (npml < 2 || npml > 1023) {
        for (i = 0; i < nx * ny; i++) { coef[i] = 1.0f; passes[i] = 0; }
        return;
    }
    a = sqrt(-log(amp) / ((npml - 1) * (npml - 1)));
    for (p = 1; p <= npml; p++) c[p] = exp(-(a * a * (npml - p) * (npml - p)));
    for (i = 0; i < nx * ny; i++) { coef[i] = 1.0f; passes[i] = 0; }
#define COEF(jj, ii) coef[((jj) - 1) * nx + (ii) - 1]
#define PASS(jj, ii) passes[((jj) - 1) * nx + (ii) - 1]
    for (p = 1; p <= npml; p++) for (j = p; j <= ny - p + 1; j++) COEF(j, p) = c[p];
    for (p = 1; p <= npml; p++) for (j = p; j <= ny - p + 1; j++) COEF(j, nx - p + 1) = c[p];
    if (free_surf == 0)
        for (p = 1; p <= npml; p++) for (i = p; i <= nx - p + 1; i++) COEF(p, i) = c[p];
    for (p = 1; p <= npml; p++) for (i = p; i <= nx - p + 1; i++) COEF(ny - p + 1, i) = c[p];
    for (i = 1; i <= npml; i++) for (j = 1; j <= ny; j++) PASS(j, i)++;
    for (i = npml + nx0 + 1; i <= nx; i++) for (j = 1; j <= ny; j++) PASS(j, i)++;
    if (free_surf == 0) for (i = 1; i <= nx; i++) for (j = 1; j <= npml; j++) PASS(j, i)++;
    for (i = 1; i <= nx; i++) for (j = fsshift + ny0 + 1; j <= ny; j++) PASS(j, i)++;
#undef COEF
#undef PASS
}

/* Gaussian gradient filter of gauss_filt (src/gauss_filt.c:27-118): half
 * widths hfs[0] (x), hfs[1] (y) and the normalised (2 hfs[1] + 1) x
 * (2 hfs[0] + 1) weights w[(jj + hfsy) * (2 hfsx + 1) + ii + hfsx], in the
 * reference's float / double arithmetic and summation order.  Returns 0 when
 * the filter is off (a zero size), else the number of weights; at most
 * wmax weights are written (-1 if more are needed). */
int gmh_gauss_kernel(float dh, float vref, float fc_low, float fsg, float fsg1, int hfs[2], float *w, int wmax)
{
    float lam = vref / fc_low;
    int fsx = round((fsg * lam) / dh), fsy = round((fsg1 * lam) / dh);
    int hfsx, hfsy, ii, jj, nwx, nwy;
    float sigmax, sigmay, sx, sy, sum = 0.0;
    if (fsx == 0 || fsy == 0) return 0;
    if (!(fsx % 2)) fsx += fsx > 0 ? 1 : -1;
    if (!(fsy % 2)) fsy += fsy > 0 ? 1 : -1;
    hfsx = abs(fsx) / 2;
    sigmax = hfsx / 2;
    sx = 2.0 * sigmax * sigmax;
    hfsy = abs(fsy) / 2;
    sigmay = hfsy / 2;
    sy = 2.0 * sigmay * sigmay;
    nwx = 2 * hfsx + 1;
    nwy = 2 * hfsy + 1;
    if (nwx * nwy > wmax) return -1;
    hfs[0] = hfsx;
    hfs[1] = hfsy;
    for (ii = -hfsx; ii <= hfsx; ii++)
        for (jj = -hfsy; jj <= hfsy; jj++) {
            float *k = &w[(jj + hfsy) * nwx + ii + hfsx];
            *k = exp(-((ii * ii) / sx) - ((jj * jj) / sy));
            sum += *k;
        }
    /* the reference normalises over i <= filt_size_x, j <= filt_size_y: a
     * negative size leaves the weights unnormalised */
    if (fsx > 0 && fsy > 0)
        for (ii = 0; ii < nwx * nwy; ii++) w[ii] /= sum;
    return nwx * nwy;
}

/* ---------------------------------------------------------------------
 * Per-shot gradient tapers of ass_grad_AC / ass_grad_TE
 * (src/AC/ass_grad_AC.c:37-43, src/TE/ass_grad_TE.c:41-49), selected by
 * SWS_TAPER_CIRCULAR_PER_SHOT:
 *   1  taper_grad_shot  (src/taper_grad_shot.c:11-99): the shot's gradient
 *      times a radial taper around its source and around every receiver,
 *      f0 + (1 - f0) (1/2 - 1/2 cos(pi r / R))^a inside the radius
 *      R = SRTRADIUS, 1 outside, f0 = 1e-3, a = -log2((0.1 - f0) / (1 - f0));
 *   2  taper_grad_shot1 (src/taper_grad_shot1.c:11-60): the shot's gradient
 *      set to 1e-5 on the (2 FILTSIZE + 1)^2 squares around every source
 *      of the call and every receiver.
 * Both read the interior source coordinates (metres) and receiver grid
 * indices as if they were full-grid ones (x = ix DH over the whole grid, no
 * NPML / FSSHIFT shift): the tapers sit NPML columns (FSSHIFT rows) away
 * from the physical positions.  Reproduced.  Grids are row-major [NY][NX];
 * (ix, iy) are the reference's 1-based indices.
 * --------------------------------------------------------------------- */
static float srt_exponent(void)
{
    float frh = 0.1, f0 = 1e-3;
    return -(log(frh - f0) - log(1.0 - f0)) / log(2.0);
}

/* coefficient of the radial taper at (ix, iy) for a centre (xc, yc) in
 * metres: the reference's float / double evaluation order */
float gmh_srt_coef(int ix, int iy, float dh, float xc, float yc, float radius)
{
    const float f0 = 1e-3, a = srt_exponent();
    float x = ix * dh, y = iy * dh, r, taper = 1.0;
    r = sqrt(pow((x - xc), 2.0) + pow((y - yc), 2.0));
    if (r <= radius) taper = f0 + (1.0 - f0) * pow((0.5 - 0.5 * cos(3.141592653589793 * r / radius)), a);
    return taper;
}

/* 1-based index range [*lo, *hi] of points i with i dh within radius of c,
 * one point of margin, clamped to [1, n] (*lo > *hi: none) */
void gmh_srt_range(float c, float radius, float dh, int n, int *lo, int *hi)
{
    double l = floor((c - radius) / dh) - 1.0, h = ceil((c + radius) / dh) + 1.0;
    *lo = l < 1.0 ? 1 : (l > n ? n + 1 : (int)l);
    *hi = h > n ? n : (h < 1.0 ? 0 : (int)h);
}

/* radial taper of one centre applied to grid (float products, in place);
 * outside the window the reference multiplies by 1.0f, which changes nothing */
static void srt_apply(int nx, int ny, float dh, float xc, float yc, float radius, float *grid)
{
    int x0, x1, y0, y1, ix, iy;
    gmh_srt_range(xc, radius, dh, nx, &x0, &x1);
    gmh_srt_range(yc, radius, dh, ny, &y0, &y1);
    for (iy = y0; iy <= y1; iy++)
        for (ix = x0; ix <= x1; ix++) grid[(size_t)(iy - 1) * nx + ix - 1] *= gmh_srt_coef(ix, iy, dh, xc, yc, radius);
}

/* taper_grad_shot on one shot's float gradient: the source of shot ishot
 * (0-based) first, then the receivers in order */
void gmh_taper_grad_shot(int nx, int ny, float dh, float radius, const float *sx, const float *sy, int ntr,
                         const int *rx, const int *ry, int ishot, float *grid)
{
    int n;
    srt_apply(nx, ny, dh, sx[ishot], sy[ishot], radius, grid);
    for (n = 0; n < ntr; n++) srt_apply(nx, ny, dh, rx[n] * dh, ry[n] * dh, radius, grid);
}

/* square of taper_grad_shot1 around grid point (i1, j1), clipped to the
 * grid (the reference writes past the array when a square crosses the
 * edge); value written: mark != NULL sets mark to 1, else grid to 1e-5 */
static void square_set(int nx, int ny, int i1, int j1, int filtsize, float *grid, unsigned char *mark)
{
    int i, j;
    for (i = i1 - filtsize; i <= i1 + filtsize; i++)
        for (j = j1 - filtsize; j <= j1 + filtsize; j++) {
            if (i < 1 || i > nx || j < 1 || j > ny) continue;
            if (mark)
                mark[(size_t)(j - 1) * nx + i - 1] = 1;
            else
                grid[(size_t)(j - 1) * nx + i - 1] = 1e-5f;
        }
}

/* taper_grad_shot1 on one shot's float gradient (grid != NULL), or its
 * mask of the points it overwrites (mark != NULL, zeroed by the caller) */
void gmh_taper_grad_shot1(int nx, int ny, float dh, int filtsize, int nshots, const float *sx, const float *sy,
                          int ntr, const int *rx, const int *ry, float *grid, unsigned char *mark)
{
    int n;
    for (n = 0; n < nshots; n++) {
        float qx = sx[n] / dh, qy = sy[n] / dh;
        square_set(nx, ny, (int)floor(qx + 0.5), (int)floor(qy + 0.5), filtsize, grid, mark);
    }
    for (n = 0; n < ntr; n++) square_set(nx, ny, rx[n], ry[n], filtsize, grid, mark);
}

/* product over the receivers of their radial taper coefficients, in double
 * (prod[n] = 1 where no receiver is within reach) */
void gmh_srt_receiver_product(int nx, int ny, float dh, float radius, int ntr, const int *rx, const int *ry,
                              double *prod)
{
    int n, x0, x1, y0, y1, ix, iy;
    for (ix = 0; ix < nx * ny; ix++) prod[ix] = 1.0;
    for (n = 0; n < ntr; n++) {
        const float xc = rx[n] * dh, yc = ry[n] * dh;
        gmh_srt_range(xc, radius, dh, nx, &x0, &x1);
        gmh_srt_range(yc, radius, dh, ny, &y0, &y1);
        for (iy = y0; iy <= y1; iy++)
            for (ix = x0; ix <= x1; ix++)
                prod[(size_t)(iy - 1) * nx + ix - 1] *= (double)gmh_srt_coef(ix, iy, dh, xc, yc, radius);
    }
}

/* ---------------------------------------------------------------------
 * Tikhonov regularisation of TE FWI on the normalised models
 * s = (BETA_MAT1 / MAT1_NORM) sigma and e = (BETA_MAT2 / MAT2_NORM) epsilon
 * (scale_grad, src/scale_grad.c:10-24): the five-point Laplacian
 * L(m) = (W + E + N + S - 4 C) / DH^2 at every IDX-th column and IDY-th row
 * of the points 2 .. NX-1, 2 .. NY-1 (src/TE/Tikhonov_cost_TE.c:27-38,
 * src/TE/Tikhonov_grad_TE.c:27-36).  The neighbour sum is float, the centre
 * term double (the 4.0 literal), DH^2 a float product, the quotient stored
 * as float; the penalty sums 0.5 BETA L^2 in double per point into a float.
 * Grids are row-major [NY][NX]; (i, j) 1-based.
 * --------------------------------------------------------------------- */
static float tikh_laplace(const float *m, int nx, int i, int j, float dh)
{
#define M(jj, ii) m[(size_t)((jj) - 1) * nx + (ii) - 1]
    return (M(j, i - 1) + M(j, i + 1) + M(j - 1, i) + M(j + 1, i) - 4.0 * M(j, i)) / (dh * dh);
#undef M
}

static void tikh_normalise(const float *m, float beta, float norm, int n, float *out)
{
    const float a = beta / norm;
    int k;
    for (k = 0; k < n; k++) out[k] = a * m[k];
}

/* Tikhonov_cost_TE: returns L2 + LAMBDA_1 tikh_sigma + LAMBDA_2 tikh_epsilon
 * (L2 itself when both LAMBDAs are <= 0); work holds 2 NX NY floats */
float gmh_tikhonov_cost_te(int nx, int ny, int idx, int idy, float dh, float norm1, float norm2, float beta1,
                           float beta2, float lambda1, float lambda2, const float *sigma, const float *epsilon,
                           float l2, float *work)
{
    float *sr = work, *er = work + (size_t)nx * ny, ls, le, ts = 0.0, te = 0.0;
    int i, j;
    tikh_normalise(sigma, beta1, norm1, nx * ny, sr);
    tikh_normalise(epsilon, beta2, norm2, nx * ny, er);
    for (i = 2; i <= nx - 1; i = i + idx)
        for (j = 2; j <= ny - 1; j = j + idy) {
            ls = tikh_laplace(sr, nx, i, j, dh);
            le = tikh_laplace(er, nx, i, j, dh);
            ts += 0.5 * beta1 * ls * ls;
            te += 0.5 * beta2 * le * le;
        }
    if ((lambda1 > 0.0) || (lambda2 > 0.0)) return l2 + lambda1 * ts + lambda2 * te;
    return l2;
}

/* Tikhonov_grad_TE: grad_sigma += LAMBDA_1 BETA_MAT1 L(s), grad_epsilon +=
 * LAMBDA_2 BETA_MAT2 L(e) (float), when either LAMBDA is > 0 */
void gmh_tikhonov_grad_te(int nx, int ny, int idx, int idy, float dh, float norm1, float norm2, float beta1,
                          float beta2, float lambda1, float lambda2, const float *sigma, const float *epsilon,
                          float *grad_sigma, float *grad_epsilon, float *work)
{
    float *sr = work, *er = work + (size_t)nx * ny, ls, le;
    int i, j;
    if (!((lambda1 > 0.0) || (lambda2 > 0.0))) return;
    tikh_normalise(sigma, beta1, norm1, nx * ny, sr);
    tikh_normalise(epsilon, beta2, norm2, nx * ny, er);
    for (i = 2; i <= nx - 1; i = i + idx)
        for (j = 2; j <= ny - 1; j = j + idy) {
            ls = tikh_laplace(sr, nx, i, j, dh);
            le = tikh_laplace(er, nx, i, j, dh);
            grad_sigma[(size_t)(j - 1) * nx + i - 1] += lambda1 * beta1 * ls;
            grad_epsilon[(size_t)(j - 1) * nx + i - 1] += lambda2 * beta2 * le;
        }
}
