// K1: impedance-matrix assembly on the device (replaces init_A_AC_9p_pml,
// src/AC/init_A_AC_9p_pml.c:17-220, init_A_SH_9p_pml, src/SH/init_A_SH_9p_pml.c
// :17-222, and init_A_TE_9p_pml, src/TE/init_A_TE_9p_pml.c:21-243).
//
// Output layout (HBM): A[f][q][k] complex128, direction-major (q = NW, N,
// NE, W, C, E, SW, S, SE), k = grid index, zero where the neighbour is off
// the grid.  One thread per grid row writes nine coalesced 16-byte values;
// the kernel is HBM-bound (8-12 B in, 144 B out per row).
//
// Numerics: every coefficient is evaluated with the reference's types and
// evaluation order -- complex-float products and sums, promoted to complex
// double where a double literal (0.25, 2.0) enters -- using separately
// rounded _rn intrinsics, so the stored doubles are bit-identical to the
// reference built by gcc for x86-64 (checked by the GPU parity tests).
#include "kernels.cuh"
#include "cplx.cuh"

namespace gm {

// Per-cell, per-matrix mass factor (complex float) and stiffness (float),
// from the material model of the matrix:
//   AC: mass = Omega^2 * ivp2, ivp2 = 1/(rho vp^2)   (init_mat_AC.c:21, :71)
//       stiff = b = 1/rho                          (init_mat_AC.c:24)
//   SH: mass = Omega^2 * rho, stiff = mu = rho vs^2 (init_mat_SH.c:21)
//   TE: mass = (Omega^2 mu0) * (eps + (sigma/Omega) i) (init_A_TE_9p_pml.c:76,78)
__global__ void k_cells(int physics, int n, const float *__restrict__ m0, const float *__restrict__ m1,
                        const AsmFreq *__restrict__ fq, float2 *__restrict__ mass, float *__restrict__ stiff) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (k >= n) return;
    const AsmFreq p = fq[f];
    const size_t mo = (size_t)p.model * n;
    const float a = m0[mo + k], b = m1[mo + k];
    float2 m;
    if (physics == GM_PHYS_AC) {
        const float ivp2 = __double2float_rn(__ddiv_rn(1.0, (double)__fmul_rn(__fmul_rn(b, a), a)));
        m = rn_scale(ivp2, p.om2);
        stiff[(size_t)f * n + k] = __double2float_rn(__ddiv_rn(1.0, (double)b));
    } else if (physics == GM_PHYS_SH) {
        m = rn_scale(b, p.om2);
        stiff[(size_t)f * n + k] = __fmul_rn(__fmul_rn(b, a), a);
    } else {
        const float2 q = rn_real_div_cf(b, p.om);
        // (q) * I as gcc lowers complex-float multiplication by (0 + 1i)
        const float qi_re = __fsub_rn(__fmul_rn(q.x, 0.0f), __fmul_rn(q.y, 1.0f));
        const float qi_im = __fadd_rn(__fmul_rn(q.x, 1.0f), __fmul_rn(q.y, 0.0f));
        const float2 epse = make_float2(__fadd_rn(a, qi_re), qi_im);
        m = rn_mul(p.om2mu0, epse);
    }
    mass[(size_t)f * n + k] = m;
}

struct BVals { float pm, mp, pp, mm, p0, m0, zp, zm; };

__device__ __forceinline__ double2 qterm(double q, float2 d0, float bv, float2 d) {
    // ((q * d0) * bv) * d   -- e.g. 0.25*idh2*dy0*bmm*dym
    return rn_mul(rn_scale((double)bv, rn_scale(q, rn_up(d0))), rn_up(d));
}
__device__ __forceinline__ double2 qterm2(double q, float2 d0, float2 inner) {
    // (q * d0) * inner      -- e.g. 0.25*idh2*dy0*(bpm*dym+bmm*dym)
    return rn_mul(rn_scale(q, rn_up(d0)), rn_up(inner));
}
__device__ __forceinline__ float2 eterm(float idh2, float2 d0, float bv, float2 d) {
    // ((d0 * idh2) * bv) * d  -- e.g. dy0*idh2*bm0*dym (complex float)
    return rn_mul(rn_scale(bv, rn_scale(idh2, d0)), d);
}
__device__ __forceinline__ float2 undamp(float2 t) {
    // tmp += -damp * tmp with damp = 0.0 (init_A_AC_9p_pml.c:91)
    return rn_add(t, rn_scale(-0.0f, t));
}

__global__ void k_stencil(AsmArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (k >= a.n) return;
    const int nx = a.nx, ny = a.ny;
    const int x = k % nx, y = k / nx;     // reference i = x+1, j = y+1
    const int i = x + 1, j = y + 1;
    const float *pml = a.pml + (size_t)f * a.pml_stride;
    const float *pxr = pml, *pxi = pml + (nx + 2), *pxhr = pml + 2 * (nx + 2), *pxhi = pml + 3 * (nx + 2);
    const float *pyr = pml + 4 * (nx + 2), *pyi = pyr + (ny + 2), *pyhr = pyi + (ny + 2), *pyhi = pyhr + (ny + 2);
    const float2 dx0 = make_float2(pxr[i], pxi[i]), dy0 = make_float2(pyr[j], pyi[j]);
    const float2 dxp = make_float2(pxhr[i], pxhi[i]), dxm = make_float2(pxhr[i - 1], pxhi[i - 1]);
    const float2 dyp = make_float2(pyhr[j], pyhi[j]), dym = make_float2(pyhr[j - 1], pyhi[j - 1]);

    BVals b;
    const float *stiff = a.stiff + (size_t)f * a.n;
    if (a.physics == GM_PHYS_AC) {           // pointwise buoyancy, av_rho.c:32-48
        const float v = stiff[k];
        b.pm = b.mp = b.pp = b.mm = b.p0 = b.m0 = b.zp = b.zm = v;
    } else if (a.physics == GM_PHYS_SH) {    // averaged shear modulus, av_mu.c:12-28
        auto mu = [&](int jj, int ii) {
            jj = jj < 1 ? 1 : (jj > ny ? ny : jj);
            ii = ii < 1 ? 1 : (ii > nx ? nx : ii);
            return stiff[(jj - 1) * nx + (ii - 1)];
        };
        auto q4 = [](float s0, float s1, float s2, float s3) {
            return __double2float_rn(__dmul_rn(0.25, (double)__fadd_rn(__fadd_rn(__fadd_rn(s0, s1), s2), s3)));
        };
        auto h2 = [](float s0, float s1) { return __double2float_rn(__dmul_rn(0.5, (double)__fadd_rn(s0, s1))); };
        const float c0 = mu(j, i);
        b.pm = q4(c0, mu(j, i + 1), mu(j - 1, i), mu(j - 1, i + 1));
        b.mp = q4(c0, mu(j, i - 1), mu(j + 1, i), mu(j + 1, i - 1));
        b.pp = q4(c0, mu(j, i + 1), mu(j + 1, i), mu(j + 1, i + 1));
        b.mm = q4(c0, mu(j, i - 1), mu(j - 1, i), mu(j - 1, i - 1));
        b.p0 = h2(c0, mu(j, i + 1));
        b.m0 = h2(c0, mu(j, i - 1));
        b.zp = h2(c0, mu(j + 1, i));
        b.zm = h2(c0, mu(j - 1, i));
    } else {                                 // TE: unit weights (init_A_TE_9p_pml.c:80-214)
        b.pm = b.mp = b.pp = b.mm = b.p0 = b.m0 = b.zp = b.zm = 1.0f;
    }

    const float2 *mass = a.mass + (size_t)f * a.n;
    float2 ms[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int xx = x + q % 3 - 1, yy = y + q / 3 - 1;
        ms[q] = (xx >= 0 && xx < nx && yy >= 0 && yy < ny) ? mass[yy * nx + xx] : make_float2(0.f, 0.f);
    }
    const float wa = a.w[0], wb = a.w[1], wc = a.w[2], wd = a.w[3], we = a.w[4], idh2 = a.w[5];
    const double qd = __dmul_rn(0.25, (double)idh2), nqd = __dmul_rn(-0.25, (double)idh2);
    float2 c[9];
    // NW
    c[0] = rn_down(rn_add(rn_up(rn_scale(wc, ms[0])),
                          rn_scale((double)wd, rn_add(qterm(qd, dy0, b.mm, dym), qterm(qd, dx0, b.mm, dxm)))));
    // N
    {
        const float2 iy = rn_add(rn_scale(b.pm, dym), rn_scale(b.mm, dym));
        const float2 ix = rn_sub(rn_scale(-b.pm, dxp), rn_scale(b.mm, dxm));
        const double2 dt = rn_scale((double)wd, rn_add(qterm2(qd, dy0, iy), qterm2(qd, dx0, ix)));
        const float2 et = rn_scale(we, eterm(idh2, dy0, b.m0, dym));
        c[1] = undamp(rn_down(rn_add(rn_add(rn_up(rn_scale(wb, ms[1])), dt), rn_up(et))));
    }
    // NE
    c[2] = rn_down(rn_add(rn_up(rn_scale(wc, ms[2])),
                          rn_scale((double)wd, rn_add(qterm(qd, dy0, b.pm, dym), qterm(qd, dx0, b.pm, dxp)))));
    // W
    {
        const float2 iy = rn_sub(rn_scale(-b.mp, dyp), rn_scale(b.mm, dym));
        const float2 ix = rn_add(rn_scale(b.mp, dxm), rn_scale(b.mm, dxm));
        const double2 dt = rn_scale((double)wd, rn_add(qterm2(qd, dy0, iy), qterm2(qd, dx0, ix)));
        const float2 et = rn_scale(we, eterm(idh2, dx0, b.m0, dxm));
        c[3] = undamp(rn_down(rn_add(rn_add(rn_up(rn_scale(wb, ms[3])), dt), rn_up(et))));
    }
    // centre
    {
        const float2 sy = rn_add(rn_add(rn_add(rn_scale(b.mp, dyp), rn_scale(b.pm, dym)), rn_scale(b.pp, dyp)),
                                 rn_scale(b.mm, dym));
        const float2 sx = rn_add(rn_add(rn_add(rn_scale(b.mp, dxm), rn_scale(b.pm, dxp)), rn_scale(b.pp, dxp)),
                                 rn_scale(b.mm, dxm));
        const double2 dt = rn_scale((double)wd, rn_sub(qterm2(nqd, dy0, sy), qterm2(qd, dx0, sx)));
        const float2 e1 = rn_mul(rn_scale(idh2, rn_neg(dy0)), rn_add(rn_scale(b.zp, dyp), rn_scale(b.zm, dym)));
        const float2 e2 = rn_mul(rn_scale(idh2, dx0), rn_add(rn_scale(b.p0, dxp), rn_scale(b.m0, dxm)));
        const float2 et = rn_scale(we, rn_sub(e1, e2));
        float2 t = rn_down(rn_add(rn_add(rn_up(rn_scale(wa, ms[4])), dt), rn_up(et)));
        // tmp += damp * 4.0 * tmp with damp = 0.0 (init_A_AC_9p_pml.c:141)
        t = rn_down(rn_add(rn_up(t), rn_scale(0.0, rn_up(t))));
        c[4] = t;
    }
    // E
    {
        const float2 iy = rn_sub(rn_scale(-b.pm, dym), rn_scale(b.pp, dyp));
        const float2 ix = rn_add(rn_scale(b.pm, dxp), rn_scale(b.pp, dxp));
        const double2 dt = rn_scale((double)wd, rn_add(qterm2(qd, dy0, iy), qterm2(qd, dx0, ix)));
        const float2 et = rn_scale(we, eterm(idh2, dx0, b.p0, dxp));
        c[5] = undamp(rn_down(rn_add(rn_add(rn_up(rn_scale(wb, ms[5])), dt), rn_up(et))));
    }
    // SW
    c[6] = rn_down(rn_add(rn_up(rn_scale(wc, ms[6])),
                          rn_scale((double)wd, rn_add(qterm(qd, dy0, b.mp, dyp), qterm(qd, dx0, b.mp, dxm)))));
    // S
    {
        const float2 iy = rn_add(rn_scale(b.mp, dyp), rn_scale(b.pp, dyp));
        const float2 ix = rn_sub(rn_scale(-b.mp, dxm), rn_scale(b.pp, dxp));
        const double2 dt = rn_scale((double)wd, rn_add(qterm2(qd, dy0, iy), qterm2(qd, dx0, ix)));
        const float2 et = rn_scale(we, eterm(idh2, dy0, b.zp, dyp));
        c[7] = undamp(rn_down(rn_add(rn_add(rn_up(rn_scale(wb, ms[7])), dt), rn_up(et))));
    }
    // SE
    c[8] = rn_down(rn_add(rn_up(rn_scale(wc, ms[8])),
                          rn_scale((double)wd, rn_add(qterm(qd, dy0, b.pp, dyp), qterm(qd, dx0, b.pp, dxp)))));

    double2 *out = a.A + (size_t)f * 9 * a.n;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int xx = x + q % 3 - 1, yy = y + q / 3 - 1;
        const bool in = xx >= 0 && xx < nx && yy >= 0 && yy < ny;
        out[(size_t)q * a.n + k] = in ? make_double2((double)c[q].x, (double)c[q].y) : make_double2(0.0, 0.0);
    }
}

void launch_assemble(const AsmArgs &a, const float *m0, const float *m1, const AsmFreq *fq, float *stiff,
                     cudaStream_t st) {
    const int tpb = 256;
    dim3 grid((a.n + tpb - 1) / tpb, a.nf);
    (k_cells<<<grid, tpb, 0, st>>>(a.physics, a.n, m0, m1, fq, a.mass, stiff), note_launch());
    (k_stencil<<<grid, tpb, 0, st>>>(a), note_launch());
}

}  // namespace gm
