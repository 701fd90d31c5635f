// K7: per-shot work around the block solves, fused over all shots and
// frequencies (replaces the per-shot host loops of forward_shot_AC and
// grad_obj_AC):
//   spike sources        RHS_source_AC / RHS_source_TE (src/AC/RHS_source_AC.c:32-53)
//   receiver gather      vec2mat + calc_seis_AC (src/vec2mat.c:19-26, src/AC/calc_seis_AC.c:18-22)
//   wavefield export     vec2mat layout, [nf][nshots][N] complex64 (tiled transpose)
//   residual + misfit    calc_res_AC (src/AC/calc_res_AC.c:10-95)
//   adjoint sources      RHS_source_AC_adj (src/AC/RHS_source_AC_adj.c:17-34)
//   gradient stack       ass_grad_AC / ass_grad_TE + cp_grad_frame (PML taper)
// All wavefield reads honour the reference's vec2mat one-slot shift: the
// value used at grid point k is x[k+1], and x[N] is defined as 0.
#include "kernels_epi.cuh"
#include "cplx.cuh"

namespace gm {

__global__ void k_spikes(double2 *b, int n, int nf, int ns, const int *ksrc, const double2 *amp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nf * ns) return;
    const int f = t / ns, s = t % ns;
    b[((size_t)f * n + ksrc[s]) * ns + s] = amp[f];
}

void launch_spikes(double2 *b, int n, int nf, int ns, const int *ksrc, const double2 *amp, cudaStream_t st) {
    cudaMemsetAsync(b, 0, (size_t)nf * n * ns * sizeof(double2), st);
    (k_spikes<<<(nf * ns + 255) / 256, 256, 0, st>>>(b, n, nf, ns, ksrc, amp), note_launch());
}

__device__ __forceinline__ double2 shifted(const double2 *x, int n, int ns, int k, int s) {
    // vec2mat: field value of grid point k is x[k + 1]; x[n] is defined as 0
    return (k + 1 < n) ? x[(size_t)(k + 1) * ns + s] : make_double2(0.0, 0.0);
}

// seis[f][s][t] (complex64 out) and cal[f][s][t] (complex128, optional)
__global__ void k_gather_seis(const double2 *x, int n, int nf, int ns, int ntr, const int *krec, float2 *seis,
                              double2 *cal) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t tot = (size_t)nf * ns * ntr;
    if (t >= tot) return;
    const int r = (int)(t % ntr);
    const int s = (int)((t / ntr) % ns);
    const int f = (int)(t / ((size_t)ntr * ns));
    const double2 v = shifted(x + (size_t)f * n * ns, n, ns, krec[r], s);
    if (seis) seis[t] = make_float2((float)v.x, (float)v.y);
    if (cal) cal[t] = v;
}

void launch_gather_seis(const double2 *x, int n, int nf, int ns, int ntr, const int *krec, float2 *seis, double2 *cal,
                        cudaStream_t st) {
    const size_t tot = (size_t)nf * ns * ntr;
    if (!tot) return;
    (k_gather_seis<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(x, n, nf, ns, ntr, krec, seis, cal), note_launch());
}

// field[f][s][k] = (complex64) x[f][k+1][s]: 32 x 32 tiles through shared memory
__global__ void k_field(const double2 *x, int n, int ns, float2 *field) {
    __shared__ float2 tile[32][33];
    const int f = blockIdx.z;
    const int k0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    const double2 *xf = x + (size_t)f * n * ns;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int k = k0 + j, s = s0 + threadIdx.x;
        if (k < n && s < ns) {
            const double2 v = shifted(xf, n, ns, k, s);
            tile[j][threadIdx.x] = make_float2((float)v.x, (float)v.y);
        }
    }
    __syncthreads();
    float2 *ff = field + (size_t)f * ns * n;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int s = s0 + j, k = k0 + threadIdx.x;
        if (k < n && s < ns) ff[(size_t)s * n + k] = tile[threadIdx.x][j];
    }
}

void launch_field(const double2 *x, int n, int nf, int ns, float2 *field, cudaStream_t st) {
    dim3 grid((n + 31) / 32, (ns + 31) / 32, nf);
    (k_field<<<grid, dim3(32, 8), 0, st>>>(x, n, ns, field), note_launch());
}

// Residuals of one (frequency, shot) per CTA: optional Wiener source
// estimate, MISFIT 1/2/3 (INVMAT = 1) or the observed data itself
// (INVMAT = 2, the RTM branch of calc_res_AC.c:77), the reference's zeroing
// of the adjoint source where both observed parts are below 1e-20, and the
// misfit partial sum (counted before the zeroing, as calc_res_AC.c:82-88
// does).
__global__ void k_residual_shot(const double2 *cal, const float2 *obs, int ntr, int stf_inv, int misfit,
                                int invmat, int zeroing, double2 *res, double *l2, double2 *stf) {
    const int fs = blockIdx.x;
    const double2 *c = cal + (size_t)fs * ntr;
    const float2 *o = obs + (size_t)fs * ntr;
    double2 *rs = res + (size_t)fs * ntr;
    __shared__ double red[3][256];
    double2 w = make_double2(1.0, 0.0);
    if (stf_inv) {
        double nr = 0, ni = 0, dr = 0;
        for (int t = threadIdx.x; t < ntr; t += blockDim.x) {
            const double2 cv = c[t];
            const double2 ov = make_double2(o[t].x, o[t].y);
            // conj(cal) * obs and conj(obs) * obs
            nr += cv.x * ov.x + cv.y * ov.y;
            ni += cv.x * ov.y - cv.y * ov.x;
            dr += ov.x * ov.x + ov.y * ov.y;
        }
        red[0][threadIdx.x] = nr; red[1][threadIdx.x] = ni; red[2][threadIdx.x] = dr;
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h)
                for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + h];
            __syncthreads();
        }
        w = make_double2(red[0][0] / red[2][0], red[1][0] / red[2][0]);
        __syncthreads();
    }
    const double wabs = sqrt(w.x * w.x + w.y * w.y);
    double acc = 0;
    for (int t = threadIdx.x; t < ntr; t += blockDim.x) {
        const double2 cv = c[t];
        const double2 ov = make_double2(o[t].x, o[t].y);
        double2 r;
        if (invmat == 2) {
            r = ov;
        } else if (misfit == 2) {
            // clog(obs) - clog(cal)
            r = make_double2(log(hypot(ov.x, ov.y)) - log(hypot(cv.x, cv.y)), atan2(ov.y, ov.x) - atan2(cv.y, cv.x));
        } else if (misfit == 3) {
            r = make_double2(atan2(cv.y, cv.x) - atan2(ov.y, ov.x), 0.0);
        } else {
            const double2 wc = cmul(w, cv);
            r = make_double2((ov.x - wc.x) / wabs, (ov.y - wc.y) / wabs);
        }
        acc += r.x * r.x + r.y * r.y;
        if (zeroing && o[t].x < 1e-20f && o[t].y < 1e-20f) r = make_double2(0.0, 0.0);
        rs[t] = r;
    }
    red[0][threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[0][threadIdx.x] += red[0][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        l2[fs] = red[0][0];
        stf[fs] = w;
    }
}

void launch_residual_shot(const double2 *cal, const float2 *obs, int nfs, int ntr, int stf_inv, int misfit,
                          int invmat, int zeroing, double2 *res, double *l2, double2 *stf, cudaStream_t st) {
    (k_residual_shot<<<nfs, 256, 0, st>>>(cal, obs, ntr, stf_inv, misfit, invmat, zeroing, res, l2, stf),
     note_launch());
}

// Adjoint sources conj(res)/DH^2 at the receivers; receivers sharing a grid
// point overwrite in receiver order (last one wins), as the reference's
// assignment loop does.  One thread per (frequency, shot).
__global__ void k_adjoint_src(double2 *b, int n, int nf, int ns, int ntr, const int *kadj, const double2 *res,
                              double dh2) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nf * ns) return;
    const int f = t / ns, s = t % ns;
    const double2 *r = res + (size_t)t * ntr;
    double2 *bf = b + (size_t)f * n * ns;
    for (int q = 0; q < ntr; ++q) bf[(size_t)kadj[q] * ns + s] = make_double2(r[q].x / dh2, -r[q].y / dh2);
}

void launch_adjoint_src(double2 *b, int n, int nf, int ns, int ntr, const int *kadj, const double2 *res, double dh2,
                        cudaStream_t st) {
    cudaMemsetAsync(b, 0, (size_t)nf * n * ns * sizeof(double2), st);
    (k_adjoint_src<<<(nf * ns + 127) / 128, 128, 0, st>>>(b, n, nf, ns, ntr, kadj, res, dh2), note_launch());
}

// Gradient stack over all frequencies and shots, one thread per grid point,
// FP64 accumulation, then the PML frame taper (coef^passes).
//   AC: g += -2 Re(Om2_f * u_fs * lambda_fs * stfu_fs / (rho vp^3))
//   TE: g0 += Re(stfu * u * (i Om_f) * lambda), g1 += Re(Om2_f * stfu * u * lambda)
__global__ void k_gradient(GradArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    double g0 = 0.0, g1 = 0.0;
    double mat = 0.0;
    if (!a.te) {
        const double vp = a.m0[k], rho = a.m1[k];
        mat = 1.0 / (rho * vp * vp * vp);
    }
    if (a.shot_taper == 0) {
        for (int f = 0; f < a.nf; ++f) {
            const double2 om2 = a.om2[f], om = a.om[f];
            const double2 *xf = a.xf + (size_t)f * a.n * a.ns;
            const double2 *xa = a.xa + (size_t)f * a.n * a.ns;
            for (int s = 0; s < a.ns; ++s) {
                const double2 u = shifted(xf, a.n, a.ns, k, s);
                const double2 l = shifted(xa, a.n, a.ns, k, s);
                const double2 w = a.stfu[(size_t)f * a.ns + s];
                const double2 wul = cmul(cmul(w, u), l);
                if (!a.te) {
                    g0 += -2.0 * cmul(om2, wul).x * mat;
                } else {
                    g0 += cmul(wul, make_double2(-om.y, om.x)).x;   // (i Omega) = (-Om.im, Om.re)
                    g1 += cmul(om2, wul).x;
                }
            }
        }
    } else {
        // each shot's term times its taper: radial coefficients (the shot's
        // source window, else 1, times the receivers' product), or 1e-5 in
        // place of the term on the squares
        const int ix = k % a.nx, iy = k / a.nx;
        const double crec = a.shot_taper == 1 ? a.taper_rec[k] : 1.0;
        const bool square = a.shot_taper == 2 && a.taper_mask[k];
        for (int f = 0; f < a.nf; ++f) {
            const double2 om2 = a.om2[f], om = a.om[f];
            const double2 *xf = a.xf + (size_t)f * a.n * a.ns;
            const double2 *xa = a.xa + (size_t)f * a.n * a.ns;
            for (int s = 0; s < a.ns; ++s) {
                const double2 u = shifted(xf, a.n, a.ns, k, s);
                const double2 l = shifted(xa, a.n, a.ns, k, s);
                const double2 w = a.stfu[(size_t)f * a.ns + s];
                const double2 wul = cmul(cmul(w, u), l);
                double t0, t1 = 0.0;
                if (!a.te) {
                    t0 = -2.0 * cmul(om2, wul).x * mat;
                } else {
                    t0 = cmul(wul, make_double2(-om.y, om.x)).x;
                    t1 = cmul(om2, wul).x;
                }
                if (a.shot_taper == 1) {
                    const int4 win = a.taper_win[s];
                    const int dx = ix - win.x, dy = iy - win.y;
                    const double c = (dx >= 0 && dx < win.z && dy >= 0 && dy < win.w)
                                         ? crec * (double)a.taper_src[a.taper_off[s] + dy * win.z + dx]
                                         : crec;
                    t0 *= c;
                    t1 *= c;
                } else if (square) {
                    t0 = (double)1e-5f;
                    t1 = (double)1e-5f;
                }
                g0 += t0;
                g1 += t1;
            }
        }
    }
    const float c = a.frame[k];
    const int p = a.passes[k];
    for (int q = 0; q < p; ++q) { g0 *= c; g1 *= c; }
    a.g0[k] = g0;
    if (a.te) a.g1[k] = g1;
}

void launch_gradient(const GradArgs &a, cudaStream_t st) {
    (k_gradient<<<(a.n + 127) / 128, 128, 0, st>>>(a), note_launch());
}

// Exact discrete FWI gradient of the acoustic engine (GM_OP_EXACT): the
// derivative of J = 0.5 sum |d - u(rec)|^2 over all shots and frequencies,
// with A u = s and A^T lambda = sum_rec conj(r) e_rec, with respect to vp at
// grid point c.  vp enters A only through the mass term of column c,
// A[c - off(q)][c] += w_q Omega^2 ivp2[c] (w_q = a, b, c of
// init_A_AC_9p_pml for the centre, edge and corner neighbours), so
//   dJ/divp2_c = Re(Omega^2 u_c sum_q w_q lambda_{c - off(q)}),
//   dJ/dvp_c   = dJ/divp2_c * (-2 / (rho_c vp_c^3)),
// read without the vec2mat shift; then the PML frame taper.  om2 holds the
// assembly's Omega^2 per frequency, w the three mass weights.
__global__ void k_gradient_exact(GradArgs a, double wa, double wb, double wc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    const int nx = a.nx, ny = a.n / nx, x = k % nx, y = k / nx;
    double g = 0.0;
    for (int f = 0; f < a.nf; ++f) {
        const double2 om2 = a.om2[f];
        const double2 *xf = a.xf + (size_t)f * a.n * a.ns;
        const double2 *xa = a.xa + (size_t)f * a.n * a.ns;
        for (int s = 0; s < a.ns; ++s) {
            double2 ls = make_double2(0.0, 0.0);
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const int xx = x - (q % 3 - 1), yy = y - (q / 3 - 1);   // row k' with k' + off(q) = k
                if (xx < 0 || xx >= nx || yy < 0 || yy >= ny) continue;
                const double w = q == 4 ? wa : (q & 1) ? wb : wc;
                const double2 l = xa[(size_t)(yy * nx + xx) * a.ns + s];
                ls.x += w * l.x;
                ls.y += w * l.y;
            }
            g += cmul(cmul(om2, xf[(size_t)k * a.ns + s]), ls).x;
        }
    }
    const double vp = a.m0[k], rho = a.m1[k];
    g *= -2.0 / (rho * vp * vp * vp);
    const float c = a.frame[k];
    const int p = a.passes[k];
    for (int q = 0; q < p; ++q) g *= c;
    a.g0[k] = g;
}

void launch_gradient_exact(const GradArgs &a, const float w[3], cudaStream_t st) {
    (k_gradient_exact<<<(a.n + 127) / 128, 128, 0, st>>>(a, w[0], w[1], w[2]), note_launch());
}

// sq[f][k] (+)= sum_s |field(k)|^2 over the ns solutions of frequency f, the
// field read through the vec2mat shift: the |F|^2 (shots) and |G|^2
// (receiver Green's functions) factors of the diagonal Hessians.
__global__ void k_hess_sq(const double2 *__restrict__ x, int n, int nf, int ns, double *sq, int accumulate) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nf * n) return;
    const int k = (int)(t % n), f = (int)(t / n);
    double acc = 0.0;
    if (k + 1 < n) {
        const double2 *row = x + ((size_t)f * n + k + 1) * ns;
        for (int s = 0; s < ns; ++s) {
            const double2 v = __ldg(row + s);
            acc += v.x * v.x + v.y * v.y;
        }
    }
    sq[t] = accumulate ? sq[t] + acc : acc;
}

void launch_hess_sq(const double2 *x, int n, int nf, int ns, double *sq, int accumulate, cudaStream_t st) {
    const size_t tot = (size_t)nf * n;
    (k_hess_sq<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(x, n, nf, ns, sq, accumulate), note_launch());
}

// h0/h1[k] = taper^passes * sum_f w_f * sqf[f][k] (* sqg[f][k]) (* mat^2):
// |J|^2 of hessian_shin_AC / hessian_AC and the TE twins summed over shots
// (and receivers), with |a F G|^2 = |a|^2 |F|^2 |G|^2 so the shot and
// receiver sums factor.
__global__ void k_hess_final(HessArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    double h0 = 0.0, h1 = 0.0;
    for (int f = 0; f < a.nf; ++f) {
        double v = a.sqf[(size_t)f * a.n + k];
        if (a.sqg) v *= a.sqg[(size_t)f * a.n + k];
        h0 += a.w0[f] * v;
        if (a.te) h1 += a.w1[f] * v;
    }
    if (!a.te) {
        const double vp = a.m0[k], rho = a.m1[k];
        const double mat = 1.0 / (rho * vp * vp * vp);
        h0 *= mat * mat;
    }
    // the float output follows the reference's order: the Hessian is a float
    // array when cp_grad_frame tapers it, so a frame point whose untapered
    // sum exceeds the float range is inf there, as in the reference
    const float c = a.frame[k];
    const int p = a.passes[k];
    float v0 = __double2float_rn(h0), v1 = __double2float_rn(h1);
    for (int q = 0; q < p; ++q) {
        h0 *= c; h1 *= c;
        v0 = __fmul_rn(v0, c); v1 = __fmul_rn(v1, c);
    }
    a.h0[k] = h0;
    a.f0[k] = v0;
    if (a.te) {
        a.h1[k] = h1;
        a.f1[k] = v1;
    }
}

void launch_hess_final(const HessArgs &a, cudaStream_t st) {
    (k_hess_final<<<(a.n + 127) / 128, 128, 0, st>>>(a), note_launch());
}

}  // namespace gm
