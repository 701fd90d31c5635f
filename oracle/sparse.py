"""TEST ORACLE: FP64 sparse direct solves and FP64 restatements of the
per-shot arithmetic (test infrastructure only; see oracle/__init__.py).

UMFPACK (SuiteSparse, not vendored in the reference and with no pinned
version; linked as ``-lumfpack`` at src/Makefile:32) is restated by SciPy's
SuperLU (``scipy.sparse.linalg.splu``, complex128), applied to the operator
UMFPACK actually factorises: the drivers build CSC structure with
umfpack_zi_triplet_to_col and then overwrite the values with the row-major
triplet order (src/AC/forward_shot_AC.c:41-48), so UMFPACK sees M = A^T where
A has the assembled stencils as rows.  UMFPACK_A solves M x = b
(forward_shot_AC.c:88, grad_obj_AC.c:121,147), UMFPACK_Aat solves
M^T x = b (grad_obj_TE.c:149).

The FP64 restatements of vec2mat (src/vec2mat.c:19-26), calc_seis_AC
(src/AC/calc_seis_AC.c:18-22), calc_res_AC (src/AC/calc_res_AC.c:10-95),
RHS_source_AC_adj (src/AC/RHS_source_AC_adj.c:17-34), ass_grad_AC/TE
(src/AC/ass_grad_AC.c:22-52, src/TE/ass_grad_TE.c:22-59) and cp_grad_frame
(src/cp_grad_frame.c:108-214) keep the reference's index conventions
(one-slot vec2mat shift, receiver/adjoint indices, residual zeroing) but
evaluate in double instead of float.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import PHYS_TE, Grid, Port


def iround_div(x: float, dh: float) -> int:
    q = np.float32(np.float32(x) / np.float32(dh))
    return int(np.floor(np.float64(q) + 0.5))


def source_index(g: Grid, xs: float, ys: float) -> int:
    """RHS index of a spike source (src/AC/RHS_source_AC.c:24-32)."""
    return (iround_div(xs, g.dh) + g.npml) + (iround_div(ys, g.dh) + g.fsshift - 1) * g.nx


def receiver_read_index(g: Grid, rx: int, ry: int) -> int:
    """Flat index into the vec2mat field read by calc_seis_AC."""
    return (ry + g.fsshift - 1) * g.nx + (rx + g.npml - 1)


def adjoint_index(g: Grid, rx: int, ry: int) -> int:
    return (rx + g.npml) + (ry + g.fsshift - 1) * g.nx


def assembled_matrix(g: Grid, ar, ai, ir, ic) -> sp.csr_matrix:
    """A with row k = stencil of grid point k (the triplets as assembled)."""
    return sp.csr_matrix((ar + 1j * ai, (ir, ic)), shape=(g.n, g.n))


def operator(A: sp.csr_matrix, op_mode: int = 0) -> sp.csc_matrix:
    """op_mode 0 (REF): M = A^T, the matrix UMFPACK factorises; 1 (EXACT): M = A."""
    return (A.T if op_mode == 0 else A).tocsc()


class DirectSolver:
    """SuperLU factorisation of M with UMFPACK_A / UMFPACK_Aat solves."""

    def __init__(self, M: sp.csc_matrix):
        self.M = M
        self.lu = spla.splu(M, permc_spec="COLAMD")

    def solve(self, b, trans: bool = False):
        return self.lu.solve(np.asarray(b, np.complex128), trans="T" if trans else "N")


def vec2mat(x: np.ndarray) -> np.ndarray:
    """FP64 vec2mat: field[k] = x[k+1], x[n] := 0 (complex128)."""
    f = np.zeros_like(x)
    f[..., :-1] = x[..., 1:]
    return f


def spike_rhs(g: Grid, physics: int, freq: float, xs, ys, port: Port | None = None) -> np.ndarray:
    """[n][nshots] complex128 right-hand sides (RHS_source_AC / RHS_source_TE)."""
    port = port or Port(g)
    ns = len(xs)
    B = np.zeros((g.n, ns), np.complex128)
    for s in range(ns):
        rr, ri = port.rhs_source(physics, freq, float(xs[s]), float(ys[s]))
        B[:, s] = rr + 1j * ri
    return B


def residual_fp64(cal, obs, stf_inv: int = 0, misfit: int = 1, invmat: int = 1):
    """calc_res_AC in double for one shot: returns (l2, res, wien); invmat 2
    is the RTM branch (residual = observed data, src/AC/calc_res_AC.c:77)."""
    cal = np.asarray(cal, np.complex128)
    obs_c = np.asarray(obs, np.complex64)
    o = obs_c.astype(np.complex128)
    w = 1.0 + 0j
    if stf_inv:
        w = np.sum(np.conj(cal) * o) / np.sum(np.conj(o) * o)
    if invmat == 2:
        res = o.copy()
    elif misfit == 1:
        res = (o - w * cal) / abs(w)
    elif misfit == 2:
        res = np.log(o) - np.log(cal)
    else:
        res = (np.angle(cal) - np.angle(o)).astype(np.complex128)
    l2 = float(np.sum((res * np.conj(res)).real))
    res = res.copy()
    zero = (obs_c.real < np.float32(1e-20)) & (obs_c.imag < np.float32(1e-20))
    res[zero] = 0
    return l2, res, w


def grad_frame(g: Grid, port: Port | None = None):
    """Coefficient field and per-point multiplicity of cp_grad_frame's taper."""
    port = port or Port(g)
    coef = port.grad_frame_coeff().astype(np.float64)
    nx, ny, npml, fs = g.nx, g.ny, g.npml, g.fsshift
    nx0, ny0 = nx - 2 * npml, ny - npml - fs
    passes = np.zeros((ny, nx), np.int32)
    passes[:, :npml] += 1
    passes[:, npml + nx0:] += 1
    if g.free_surf == 0:
        passes[:npml, :] += 1
    passes[fs + ny0:, :] += 1
    return coef, passes.reshape(-1)


def shot_taper(g: Grid, mode: int, sx, sy, rx, ry, radius: float = 0.0, filtsize: int = 0,
               port: Port | None = None):
    """The per-shot gradient taper of ass_grad_AC / ass_grad_TE
    (SWS_TAPER_CIRCULAR_PER_SHOT, src/AC/ass_grad_AC.c:37-43) in the FP64
    form the gradient stack applies: mode 1 ("radial", C[ns][n]) with
    C_s = (product over the receivers, in order, of their radial
    coefficients) * (shot s's source coefficients), the coefficients those
    of taper_grad_shot (port_srt_field); mode 2 ("squares", mask[n]) with
    the points taper_grad_shot1 overwrites; mode 0 None."""
    port = port or Port(g)
    if mode == 1:
        dh = np.float32(g.dh)
        crec = np.ones(g.n)
        for x, y in zip(rx, ry):
            crec *= port.srt_field(np.float32(x) * dh, np.float32(y) * dh, radius).astype(np.float64)
        C = np.stack([crec * port.srt_field(float(sx[s]), float(sy[s]), radius).astype(np.float64)
                      for s in range(len(sx))])
        return ("radial", C)
    if mode == 2:
        return ("squares", port.taper_grad_shot1(np.zeros(g.n, np.float32), filtsize, sx, sy, rx, ry) != 0)
    return None


def _taper_terms(t, taper):
    """Per-shot terms [ns][n] of one frequency after the shot taper."""
    if taper is None:
        return t
    kind, val = taper
    if kind == "radial":
        return t * val
    t = t.copy()
    t[:, val] = float(np.float32(1e-5))
    return t


def gradient_fp64(g: Grid, physics: int, freqs, Xf, Xa, stfu, vp=None, rho=None, port: Port | None = None,
                  taper=None):
    """FP64 ass_grad_AC / ass_grad_TE summed over frequencies and shots, then
    the cp_grad_frame taper.  Xf, Xa: [nf][n][ns] solutions; stfu[nf][ns];
    taper: the per-shot taper of shot_taper (None: SWS_TAPER_CIRCULAR_PER_SHOT
    = 0)."""
    port = port or Port(g)
    nf = len(freqs)
    g0 = np.zeros(g.n)
    g1 = np.zeros(g.n)
    mat = None
    if physics != PHYS_TE:
        vpd = np.asarray(vp, np.float64).reshape(-1)
        rhod = np.asarray(rho, np.float64).reshape(-1)
        mat = 1.0 / (rhod * vpd ** 3)
    for f in range(nf):
        om2, om = port.gradient_scalars(physics, float(freqs[f]))
        u = vec2mat(Xf[f].T)  # [ns][n]
        lam = vec2mat(Xa[f].T)
        wul = stfu[f][:, None] * u * lam
        if taper is None and physics != PHYS_TE:
            g0 += np.sum(-2.0 * (om2 * wul).real * mat[None, :], axis=0)
        elif taper is None:
            g0 += np.sum((wul * (1j * om)).real, axis=0)
            g1 += np.sum((om2 * wul).real, axis=0)
        elif physics != PHYS_TE:
            g0 += np.sum(_taper_terms(-2.0 * (om2 * wul).real * mat[None, :], taper), axis=0)
        else:
            g0 += np.sum(_taper_terms((wul * (1j * om)).real, taper), axis=0)
            g1 += np.sum(_taper_terms((om2 * wul).real, taper), axis=0)
    coef, passes = grad_frame(g, port)
    fac = coef ** passes
    return g0 * fac, (g1 * fac if physics == PHYS_TE else None)


def hess_green_rhs(g: Grid, physics: int, rx, ry) -> np.ndarray:
    """[n][ntr] right-hand sides of the Hessian's receiver Green's functions:
    a spike at the adjoint index (RHS_source_AC_hess, src/AC/RHS_source_AC_hess.c:26-33:
    float amp 1 over float DH*DH; RHS_source_TE_hess, src/TE/RHS_source_TE_hess.c:34-38:
    1.0 / (DH*DH) in double)."""
    dh2 = np.float32(g.dh) * np.float32(g.dh)
    amp = float(1.0 / np.float64(dh2)) if physics == PHYS_TE else float(np.float32(1.0) / dh2)
    B = np.zeros((g.n, len(rx)), complex)
    for t, (a, b) in enumerate(zip(rx, ry)):
        B[adjoint_index(g, int(a), int(b)), t] = amp
    return B


def hessian_source_physics(physics: int, mode: int) -> int:
    """The physics whose source routine models the Hessian's forward fields:
    hessian_shin_TE calls RHS_source_AC (src/TE/hessian_shin_TE.c:108, a
    1/DH^2 spike without the -i Omega mu0 of RHS_source_TE); every other
    estimator uses its own physics' source."""
    return 1 if (physics == PHYS_TE and mode == 2) else physics


def hessian_fp64(g: Grid, physics: int, mode: int, freqs, Xf, Xg=None, vp=None, rho=None,
                 port: Port | None = None, tapered: bool = True):
    """FP64 diagonal Hessians term by term, then the cp_grad_frame taper:
    mode 2, hessian_shin_AC (src/AC/hessian_shin_AC.c:117-126):
        sum_s |J|^2, J = 2 Omega^2 F_s / (rho vp^3);
    mode 1, hessian_AC (src/AC/hessian_AC.c:152-160):
        sum_s sum_r |J|^2, J = -2 Omega^2 F_s G_r / (rho vp^3);
    TE (src/TE/hessian_shin_TE.c:121-128, src/TE/hessian_TE.c:147-158):
        sigma J = (i Omega) F_s (G_r), epsilon J = Omega^2 F_s (G_r).
    Xf: [nf][n][ns] forward solutions, Xg: [nf][n][ntr] Green's functions
    (both before the vec2mat shift).  Returns (h0, h1) [n]; h1 None for AC;
    tapered=False leaves out the cp_grad_frame taper."""
    port = port or Port(g)
    h0 = np.zeros(g.n)
    h1 = np.zeros(g.n)
    mat = None
    if physics != PHYS_TE:
        vpd = np.asarray(vp, np.float64).reshape(-1)
        rhod = np.asarray(rho, np.float64).reshape(-1)
        mat = 1.0 / (rhod * vpd ** 3)
    for f in range(len(freqs)):
        om2, om = port.gradient_scalars(physics, float(freqs[f]))
        F = vec2mat(Xf[f].T)                                   # [ns][n]
        G = vec2mat(Xg[f].T) if mode == 1 else np.ones((1, g.n))   # [ntr][n]
        FG = F[:, None, :] * G[None, :, :]                      # [ns][ntr][n], one term per (shot, receiver)
        if physics != PHYS_TE:
            J = (-2.0 if mode == 1 else 2.0) * om2 * FG * mat
            h0 += np.sum(np.abs(J) ** 2, axis=(0, 1))
        else:
            h0 += np.sum(np.abs(1j * om * FG) ** 2, axis=(0, 1))
            h1 += np.sum(np.abs(om2 * FG) ** 2, axis=(0, 1))
    if not tapered:
        return h0, (h1 if physics == PHYS_TE else None)
    coef, passes = grad_frame(g, port)
    fac = coef ** passes
    return h0 * fac, (h1 * fac if physics == PHYS_TE else None)


def taper_float(g: Grid, h, port: Port | None = None) -> np.ndarray:
    """cp_grad_frame on a float array (src/cp_grad_frame.c:162-200): the
    untapered sum rounded to float, then multiplied in float by the taper
    coefficient once per boundary strip the point lies in."""
    coef, passes = grad_frame(g, port or Port(g))
    v = np.asarray(h, np.float64).astype(np.float32)
    c = np.asarray(coef, np.float32)
    for q in range(int(np.max(passes)) if np.size(passes) else 0):
        sel = passes > q
        v[sel] = v[sel] * c[sel]
    return v
