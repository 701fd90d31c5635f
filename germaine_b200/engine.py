"""Host-side mirror of GERMAINE's per-frequency engine over the C-ABI.

The reference drives one frequency at a time through
``forward_shot_AC`` (src/AC/forward_shot_AC.c:10), ``grad_obj_AC``
(src/AC/grad_obj_AC.c:10) and ``obj_AC`` (src/AC/obj_AC.c:10) (TE/SH twins
alike), each of which assembles the impedance matrix, factorises it with
UMFPACK and loops over the shots.  :class:`Engine` exposes the same steps
over libgermaine_gpu.so, batched over frequencies and shots: ``factor``
(assembly + numeric LU of every frequency of a stage), then ``forward`` /
``grad_obj`` / ``obj`` over all shots at once, and ``solve`` for arbitrary
right-hand sides (the ``umfpack_zi_solve`` level).

Argument meaning follows the reference: grids are the full NX x NY grid with
the PML frame (forward_AC.c:44-45), source positions are in metres
(srcpos[1]/[2]), receiver positions are grid indices without the PML offset
(recpos[1]/[2]), seismograms use the reference's flat index
``i + ntr*(ishot-1) + ntr*nshots*(nfreq-1)``.  Errors raise
:class:`~germaine_b200._lib.GmError`; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (GM_OP_EXACT, GM_OP_REF, GM_PHYS_AC, GM_PHYS_SH, GM_PHYS_TE, GM_PREC_C64_IR, GM_PREC_FP64,
                   GM_SYS_A, GM_SYS_AT, GmConfig, GmStats, check, ptr)

__all__ = ["Engine", "gauss_filt", "GM_PHYS_AC", "GM_PHYS_SH", "GM_PHYS_TE", "GM_PREC_FP64", "GM_PREC_C64_IR",
           "GM_OP_REF", "GM_OP_EXACT", "GM_SYS_A", "GM_SYS_AT", "nonzero"]


def nonzero(nx: int, ny: int) -> int:
    """NONZERO of the 9-point pattern (src/calc_nonzero.c:10-52)."""
    return 9 * nx * ny - 6 * nx - 6 * ny + 4


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Engine:
    """One GPU engine for one NX x NY grid and one physics."""

    def __init__(self, nx: int, ny: int, dh: float, npml: int, physics: int = GM_PHYS_AC,
                 precision: int = GM_PREC_FP64, op_mode: int = GM_OP_REF, free_surf: int = 0,
                 a0_pml: float = 90.0, s: float = 0.0, device: int = 0, leaf_max: int = 32,
                 ir_tol: float = 1e-10, ir_max_iter: int = 10, refine: int = 0, gmres_restart: int = 0,
                 tc_min_block: int = 0, pivot_tol: float = 0.0):
        self.lib = _lib.load()
        self.cfg = GmConfig(nx, ny, dh, npml, free_surf, a0_pml, s, physics, precision, op_mode, leaf_max,
                            ir_tol, ir_max_iter, refine, gmres_restart, tc_min_block, pivot_tol)
        self.nx, self.ny, self.n = nx, ny, nx * ny
        self.physics = physics
        self._h = ctypes.c_void_p()
        check(self.lib.gm_engine_create(device, ctypes.byref(self.cfg), ctypes.byref(self._h)))
        self.nf = 0
        self.freqs = None
        self.last_status = 0

    # -- lifetime --
    def close(self):
        if self._h:
            self.lib.gm_engine_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- set-up --
    def set_model(self, mat0, mat1):
        """Material arrays [NY][NX] (AC: vp, rho; SH: vs, rho; TE: epsilon,
        sigma): numpy arrays or torch float32 tensors (host or device)."""
        if hasattr(mat0, "data_ptr"):
            if mat0.numel() != self.n or mat1.numel() != self.n:
                raise ValueError(f"material arrays must have {self.n} entries")
            self._m = (mat0, mat1)
            check(self.lib.gm_set_model(self._h, ptr(mat0), ptr(mat1)))
            return
        m0 = _c(mat0, np.float32).reshape(-1)
        m1 = _c(mat1, np.float32).reshape(-1)
        if m0.size != self.n or m1.size != self.n:
            raise ValueError(f"material arrays must have {self.n} entries")
        self._m = (m0, m1)
        check(self.lib.gm_set_model(self._h, ptr(m0), ptr(m1)))

    def set_models(self, mat0, mat1):
        """Several material models [nmod][NY][NX] for gm_factor_models
        (line-search trial models)."""
        m0 = _c(mat0, np.float32)
        m1 = _c(mat1, np.float32)
        if m0.shape != m1.shape or m0.size % self.n:
            raise ValueError("models must be [nmod][ny][nx] pairs")
        check(self.lib.gm_set_models(self._h, m0.size // self.n, ptr(m0), ptr(m1)))

    def factor_models(self, freqs, models) -> int:
        """Factorise matrix m at freqs[m] from model models[m] (one batch)."""
        f = _c(freqs, np.float32)
        mi = _c(models, np.int32)
        if f.size != mi.size:
            raise ValueError("one model index per matrix")
        self.last_status = check(self.lib.gm_factor_models(self._h, f.size, ptr(f), ptr(mi)))
        self.nf = f.size
        self.freqs = f
        return self.last_status

    def obj_each(self, src_x, src_y, rec_x, rec_y, pobs, stf_inv: int = 0, misfit: int = 1) -> np.ndarray:
        """Misfit (0.5 L2) of every factorised matrix."""
        sx = _c(src_x, np.float32); sy = _c(src_y, np.float32)
        rx = _c(rec_x, np.int32); ry = _c(rec_y, np.int32)
        obs = _c(pobs, np.complex64).reshape(self.nf, sx.size, rx.size)
        out = np.zeros(self.nf, np.float32)
        self.last_status = check(self.lib.gm_obj_each(self._h, sx.size, ptr(sx), ptr(sy), rx.size, ptr(rx), ptr(ry),
                                                      ptr(obs), stf_inv, misfit, ptr(out)))
        return out

    def factor(self, freqs) -> int:
        f = _c(np.atleast_1d(freqs), np.float32)
        self.last_status = check(self.lib.gm_factor(self._h, int(f.size), ptr(f)))
        self.nf = int(f.size)
        self.freqs = f
        return self.last_status

    def autotune(self, nrhs: int, reps: int = 2):
        """Choose the substitution tiles of every level for nrhs right-hand
        sides by timing the candidates on the current factors (gm_autotune);
        returns the table [level] -> (fwd rows, fwd slice, bwd rows, bwd slice)."""
        check(self.lib.gm_autotune(self._h, nrhs, reps))
        nl = self.stats()["nlevels"]
        tab = np.zeros(4 * nl, np.int32)
        n = ctypes.c_int(0)
        check(self.lib.gm_autotune_table(self._h, ctypes.byref(n), ptr(tab), nl))
        return [(int(a), 8 * int(b), int(c), 8 * int(d)) for a, b, c, d in tab.reshape(nl, 4)]

    def refine_report(self) -> list[dict]:
        """Per-matrix refinement records of the last solve (gm_refine_report):
        first / final max relative residual, sweeps, method."""
        arr = (_lib.GmRefineInfo * self.nf)()
        check(self.lib.gm_refine_report(self._h, self.nf, arr))
        return [{"first_residual": a.first_residual, "final_residual": a.final_residual, "sweeps": a.sweeps,
                 "method": _lib.REFINE_METHOD_NAMES.get(a.method, str(a.method))} for a in arr]

    def stats(self) -> dict:
        s = GmStats()
        check(self.lib.gm_engine_stats(self._h, ctypes.byref(s)))
        return s.as_dict()

    def triplets(self, ifreq: int = 0):
        nz = nonzero(self.nx, self.ny)
        ar = np.zeros(nz); ai = np.zeros(nz)
        ir = np.zeros(nz, np.int32); ic = np.zeros(nz, np.int32)
        check(self.lib.gm_get_triplets(self._h, ifreq, ptr(ar), ptr(ai), ptr(ir), ptr(ic)))
        return ar, ai, ir, ic

    # -- solves --
    def solve(self, b, sys: int = GM_SYS_A):
        """b: complex array [nf][n][nrhs] (or [n][nrhs] / [n] for nf == 1)."""
        b = np.asarray(b)
        squeeze = b.ndim
        if b.ndim == 1:
            b = b[None, :, None]
        elif b.ndim == 2:
            b = b[None]
        if b.shape[0] != self.nf or b.shape[1] != self.n:
            raise ValueError(f"b must be [{self.nf}][{self.n}][nrhs]")
        bb = _c(b, np.complex128)
        x = np.empty_like(bb)
        self.last_status = check(self.lib.gm_solve(self._h, sys, int(bb.shape[2]), ptr(bb), ptr(x)))
        if squeeze == 1:
            return x[0, :, 0]
        if squeeze == 2:
            return x[0]
        return x

    def forward(self, src_x, src_y, rec_x=None, rec_y=None, want_seis: bool = True, want_field: bool = False,
                seis_out=None, field_out=None):
        """All shots of all factorised frequencies.  Returns (seis, field):
        seis [nf][nshots][ntr] complex64, field [nf][nshots][NY*NX] complex64
        in the reference's vec2mat layout (either may be None).  seis_out /
        field_out may be preallocated outputs (numpy arrays or torch tensors,
        host or device) of those shapes."""
        sx = _c(src_x, np.float32); sy = _c(src_y, np.float32)
        ns = sx.size
        rx = _c(rec_x if rec_x is not None else [], np.int32)
        ry = _c(rec_y if rec_y is not None else [], np.int32)
        ntr = rx.size
        seis = seis_out
        if seis is None and want_seis and ntr:
            seis = np.empty((self.nf, ns, ntr), np.complex64)
        field = field_out
        if field is None and want_field:
            field = np.empty((self.nf, ns, self.n), np.complex64)
        self.last_status = check(self.lib.gm_forward(self._h, ns, ptr(sx), ptr(sy), ntr, ptr(rx), ptr(ry),
                                                     ptr(seis), ptr(field)))
        return seis, field

    def stream(self) -> int:
        """Address of the CUDA stream the engine issues its work on."""
        s = ctypes.c_void_p()
        check(self.lib.gm_engine_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    def grad_obj(self, src_x, src_y, rec_x, rec_y, pobs, stf_inv: int = 0, misfit: int = 1, want_seis=False):
        """Misfit and gradient(s).  Returns (grad0, grad1, l2, seis); grad1 is
        None for AC (the reference's fwiAC.grad) and the epsilon gradient for
        TE (grad0 = sigma gradient)."""
        sx = _c(src_x, np.float32); sy = _c(src_y, np.float32)
        rx = _c(rec_x, np.int32); ry = _c(rec_y, np.int32)
        ns, ntr = sx.size, rx.size
        obs = _c(pobs, np.complex64).reshape(self.nf, ns, ntr)
        g0 = np.zeros(self.n, np.float32)
        g1 = np.zeros(self.n, np.float32) if self.physics == GM_PHYS_TE else None
        l2 = ctypes.c_float(0.0)
        seis = np.empty((self.nf, ns, ntr), np.complex64) if want_seis else None
        self.last_status = check(self.lib.gm_grad_obj(self._h, ns, ptr(sx), ptr(sy), ntr, ptr(rx), ptr(ry), ptr(obs),
                                                      stf_inv, misfit, ptr(g0), ptr(g1), ctypes.byref(l2),
                                                      ptr(seis)))
        return g0, g1, float(l2.value), seis

    def set_shot_block(self, max_shots: int) -> None:
        """Cap on shots per block solve of forward() (0: device memory decides)."""
        check(self.lib.gm_set_shot_block(self._h, max_shots))

    def set_refine(self, refine: int, gmres_restart: int = 0) -> None:
        """Refinement mode (GM_REFINE_MODE_*) and GMRES restart length of the
        following solves (0 = default)."""
        check(self.lib.gm_set_refine(self._h, refine, gmres_restart))

    def memory_estimate(self, nmat: int):
        """(bytes to factorise nmat matrices at once, bytes per shot of a block
        solve over them)."""
        fb, sb = ctypes.c_size_t(0), ctypes.c_size_t(0)
        check(self.lib.gm_memory_estimate(self._h, nmat, ctypes.byref(fb), ctypes.byref(sb)))
        return int(fb.value), int(sb.value)

    def plan(self, nfreq: int, nshots: int, budget: int):
        """Frequencies per factorisation batch and shots per block solve so that
        one batch (its factors plus one block's workspaces) fits `budget`
        device bytes; raises if even one frequency with one shot does not."""
        for nb in range(nfreq, 0, -1):
            fb, sb = self.memory_estimate(nb)
            if fb + sb <= budget:
                return nb, int(max(1, min(nshots, (budget - fb) // sb)))
        raise ValueError(f"one frequency needs {sum(self.memory_estimate(1))} bytes, more than {budget}")

    def set_invmat(self, invmat: int) -> None:
        """INVMAT of the residuals of the following grad_obj / obj calls:
        1 FWI (default), 2 RTM (residual = observed data)."""
        check(self.lib.gm_set_invmat(self._h, invmat))

    def set_source_wavelet(self, amp) -> None:
        """Per-matrix complex source amplitudes of an external wavelet
        (READ_WAVELET = 1; amp: nmat complex values, e.g. from stf_dft), or
        None for spike sources."""
        if amp is None:
            check(self.lib.gm_set_source_wavelet(self._h, 0, None))
            return
        a = _c(np.asarray(amp, np.complex64).reshape(-1).view(np.float32), np.float32)
        check(self.lib.gm_set_source_wavelet(self._h, a.size // 2, ptr(a)))

    def set_shot_taper(self, mode: int, srtradius: float = 0.0, filtsize: int = 0) -> None:
        """Per-shot gradient taper of the following grad_obj calls
        (SWS_TAPER_CIRCULAR_PER_SHOT): 0 none, 1 taper_grad_shot (radius
        SRTRADIUS in metres), 2 taper_grad_shot1 (squares of half-width
        FILTSIZE)."""
        check(self.lib.gm_set_shot_taper(self._h, mode, srtradius, filtsize))

    def wavefield_fp64(self, which: int = 0, nshots: int | None = None) -> np.ndarray:
        """FP64 solutions of the last forward-type call (which = 0) or of the
        last grad_obj's adjoint solve (which = 1): [nf][NY*NX][nshots]
        complex128 in grid order (no vec2mat shift)."""
        if nshots is None:
            raise ValueError("nshots is required")
        x = np.empty((self.nf, self.n, nshots), np.complex128)
        check(self.lib.gm_get_wavefield_fp64(self._h, which, ptr(x)))
        return x

    def misfit_fp64(self):
        """(0.5 * misfit sum, per-matrix misfits) of the last obj / obj_each /
        grad_obj, in FP64."""
        each = np.zeros(self.nf)
        l2 = ctypes.c_double(0.0)
        check(self.lib.gm_get_misfit_fp64(self._h, self.nf, ctypes.byref(l2), ptr(each)))
        return float(l2.value), each

    def gradient_fp64(self):
        g0 = np.zeros(self.n)
        g1 = np.zeros(self.n) if self.physics == GM_PHYS_TE else None
        check(self.lib.gm_get_gradient_fp64(self._h, ptr(g0), ptr(g1)))
        return g0, g1

    def hessian(self, src_x, src_y, rec_x=None, rec_y=None, mode: int = _lib.GM_HESS_SHIN):
        """Diagonal Hessian (gm_hessian): mode GM_HESS_SHIN (hessian_shin_AC,
        shots only) or GM_HESS_GREEN (hessian_AC, shots x receivers).
        Returns (hess0, hess1); hess1 is None for AC and the epsilon Hessian
        for TE (hess0 = sigma Hessian)."""
        sx = _c(src_x, np.float32); sy = _c(src_y, np.float32)
        rx = _c(rec_x if rec_x is not None else [], np.int32)
        ry = _c(rec_y if rec_y is not None else [], np.int32)
        h0 = np.zeros(self.n, np.float32)
        h1 = np.zeros(self.n, np.float32) if self.physics == GM_PHYS_TE else None
        self.last_status = check(self.lib.gm_hessian(self._h, mode, sx.size, ptr(sx), ptr(sy), rx.size, ptr(rx),
                                                     ptr(ry), ptr(h0), ptr(h1)))
        return h0, h1

    def hessian_fp64(self):
        h0 = np.zeros(self.n)
        h1 = np.zeros(self.n) if self.physics == GM_PHYS_TE else None
        check(self.lib.gm_get_hessian_fp64(self._h, ptr(h0), ptr(h1)))
        return h0, h1

    def obj(self, src_x, src_y, rec_x, rec_y, pobs, stf_inv: int = 0, misfit: int = 1) -> float:
        sx = _c(src_x, np.float32); sy = _c(src_y, np.float32)
        rx = _c(rec_x, np.int32); ry = _c(rec_y, np.int32)
        obs = _c(pobs, np.complex64).reshape(self.nf, sx.size, rx.size)
        l2 = ctypes.c_float(0.0)
        self.last_status = check(self.lib.gm_obj(self._h, sx.size, ptr(sx), ptr(sy), rx.size, ptr(rx), ptr(ry),
                                                 ptr(obs), stf_inv, misfit, ctypes.byref(l2)))
        return float(l2.value)


class Lbfgs:
    """The reference's l-BFGS update on the GPU (gm_lbfgs_*): LBFGS
    (src/LBFGS.c) for nclass = 1, LBFGS_TE (src/TE/LBFGS_TE.c) for
    nclass = 2, with the history resident on the device.  Grids are
    [nclass][NY][NX] (or [NY][NX] for one class) float32."""

    def __init__(self, nx: int, ny: int, npml: int, m: int, nclass: int = 1, free_surf: int = 0, device: int = 0):
        self.lib = _lib.load()
        self.nx, self.ny, self.nclass, self.m = nx, ny, nclass, m
        h = ctypes.c_void_p()
        check(self.lib.gm_lbfgs_create(device, nx, ny, npml, free_surf, nclass, m, ctypes.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            self.lib.gm_lbfgs_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _grid(self, a):
        g = _c(a, np.float32)
        if g.size != self.nclass * self.nx * self.ny:
            raise ValueError("grid size does not match the l-BFGS layout")
        return g

    def step(self, first: bool, pointer: int, grad, gradm, model, hess=None, eps_hess: float = 0.0):
        """One LBFGS call; returns Hgrad with the shape of gradm."""
        g, gm, md = self._grid(grad), self._grid(gradm), self._grid(model)
        hs = self._grid(hess) if hess is not None else None
        out = np.empty_like(gm)
        check(self.lib.gm_lbfgs_step(self._h, int(bool(first)), pointer, ptr(g), ptr(gm), ptr(md), ptr(hs), eps_hess,
                                     ptr(out)))
        return out

    def rotate(self):
        check(self.lib.gm_lbfgs_rotate(self._h))

    def zero(self):
        check(self.lib.gm_lbfgs_zero(self._h))

    def check_descent(self, hgrad, grad) -> float:
        """p of check_descent; the history is cleared when p < 0."""
        p = ctypes.c_float(0.0)
        check(self.lib.gm_lbfgs_check_descent(self._h, ptr(self._grid(hgrad)), ptr(self._grid(grad)),
                                              ctypes.byref(p)))
        return float(p.value)

    def get_old(self):
        shape = (self.nclass, self.ny, self.nx) if self.nclass > 1 else (self.ny, self.nx)
        g = np.empty(shape, np.float32)
        md = np.empty(shape, np.float32)
        check(self.lib.gm_lbfgs_get_old(self._h, ptr(g), ptr(md)))
        return g, md

    def set_old(self, grad_old, model_old):
        check(self.lib.gm_lbfgs_set_old(self._h, ptr(self._grid(grad_old)), ptr(self._grid(model_old))))


def mat_change(hgrad, model_old, eps_scale: float, low: float, up: float, mode: int = 0, device: int = 0):
    """calc_mat_change_wolfe (mode 0) / _multi_para (mode 1) on the GPU."""
    h = _c(hgrad, np.float32)
    old = _c(model_old, np.float32)
    out = np.empty_like(old)
    check(_lib.load().gm_mat_change(device, old.size, mode, eps_scale, low, up, ptr(h), ptr(old), ptr(out)))
    return out


def taper_grad_shot(grad, dh: float, srtradius: float, src_x, src_y, rec_x, rec_y, ishot: int) -> np.ndarray:
    """taper_grad_shot on one shot's [NY][NX] float gradient (host,
    bit-identical): returns the tapered copy; ishot is 0-based."""
    g = np.array(grad, np.float32, copy=True, order="C")
    ny, nx = g.shape
    sx = _c(src_x, np.float32); sy = _c(src_y, np.float32)
    rx = _c(rec_x, np.int32); ry = _c(rec_y, np.int32)
    check(_lib.load().gm_taper_grad_shot(nx, ny, dh, srtradius, sx.size, ptr(sx), ptr(sy), rx.size, ptr(rx),
                                         ptr(ry), ishot, ptr(g)))
    return g


def taper_grad_shot1(grad, dh: float, filtsize: int, src_x, src_y, rec_x, rec_y) -> np.ndarray:
    """taper_grad_shot1 on one shot's [NY][NX] float gradient (host,
    bit-identical): returns the tapered copy."""
    g = np.array(grad, np.float32, copy=True, order="C")
    ny, nx = g.shape
    sx = _c(src_x, np.float32); sy = _c(src_y, np.float32)
    rx = _c(rec_x, np.int32); ry = _c(rec_y, np.int32)
    check(_lib.load().gm_taper_grad_shot1(nx, ny, dh, filtsize, sx.size, ptr(sx), ptr(sy), rx.size, ptr(rx),
                                          ptr(ry), ptr(g)))
    return g


def tikhonov_cost_te(sigma, epsilon, l2: float, dh: float, mat1_norm: float, mat2_norm: float, beta_mat1: float,
                     beta_mat2: float, lambda_1: float, lambda_2: float, idx: int = 1, idy: int = 1) -> float:
    """Tikhonov_cost_TE (host, bit-identical): the misfit plus the Laplacian
    penalty of the normalised [NY][NX] sigma and epsilon models."""
    s = _c(sigma, np.float32)
    e = _c(epsilon, np.float32)
    ny, nx = np.shape(sigma)
    out = ctypes.c_float(0.0)
    check(_lib.load().gm_tikhonov_cost_te(nx, ny, idx, idy, dh, mat1_norm, mat2_norm, beta_mat1, beta_mat2, lambda_1,
                                          lambda_2, ptr(s), ptr(e), l2, ctypes.byref(out)))
    return float(out.value)


def tikhonov_grad_te(grad_sigma, grad_epsilon, sigma, epsilon, dh: float, mat1_norm: float, mat2_norm: float,
                     beta_mat1: float, beta_mat2: float, lambda_1: float, lambda_2: float, idx: int = 1,
                     idy: int = 1):
    """Tikhonov_grad_TE (host, bit-identical): returns the regularised
    copies of the two [NY][NX] TE gradients."""
    gs = np.array(grad_sigma, np.float32, copy=True, order="C")
    ge = np.array(grad_epsilon, np.float32, copy=True, order="C")
    s = _c(sigma, np.float32)
    e = _c(epsilon, np.float32)
    ny, nx = gs.shape
    check(_lib.load().gm_tikhonov_grad_te(nx, ny, idx, idy, dh, mat1_norm, mat2_norm, beta_mat1, beta_mat2, lambda_1,
                                          lambda_2, ptr(s), ptr(e), ptr(gs), ptr(ge)))
    return gs, ge


def precond(grad, npml: int, free_surf: int, dh: float, spatfilter: int = 0, vref: float = 0.0,
            fc_low: float = 1.0, filt_size_grad: float = 0.0, filt_size_grad1: float = 0.0, taper_hor: int = 0,
            gradt2: int = 0, taper=None, device: int = 0) -> np.ndarray:
    """precond() on the GPU (gm_precond: gauss_filt, taper_grad_hor,
    taper_grad_file with the "taper.bin" content given as `taper`,
    [NX0*NY0] floats x outer); returns the preconditioned copy."""
    g = np.array(grad, np.float32, copy=True, order="C")
    ny, nx = g.shape
    tp = _c(taper, np.float32) if taper is not None else None
    check(_lib.load().gm_precond(device, nx, ny, npml, free_surf, dh, spatfilter, vref, fc_low, filt_size_grad,
                                 filt_size_grad1, taper_hor, gradt2, ptr(tp), ptr(g)))
    return g


def apply_hess(grad, hess, eps_hess: float, device: int = 0):
    """apply_hess_AC on the GPU (gm_apply_hess, bit-identical): returns
    (preconditioned gradient, MAX_HESS)."""
    g = np.array(grad, np.float32, copy=True, order="C")
    h = _c(hess, np.float32)
    if g.size != h.size:
        raise ValueError("gradient and Hessian differ in size")
    mx = ctypes.c_float(0.0)
    check(_lib.load().gm_apply_hess(device, g.size, eps_hess, ptr(g), ptr(h), ctypes.byref(mx)))
    return g, float(mx.value)


def gauss_filt(grad, dh: float, vref: float, fc_low: float, filt_size_grad: float, filt_size_grad1: float,
               device: int = 0) -> np.ndarray:
    """Gaussian smoothing of a [NY][NX] gradient on the GPU (gm_gauss_filt:
    gauss_filt, src/gauss_filt.c:10-141, bit-identical)."""
    g = _c(grad, np.float32)
    ny, nx = g.shape
    out = np.empty_like(g)
    check(_lib.load().gm_gauss_filt(device, nx, ny, dh, vref, fc_low, filt_size_grad, filt_size_grad1, ptr(g),
                                    ptr(out)))
    return out


def stf_dft(path: str, physics: int, freq: float) -> complex:
    """read_stf_dft on the host (gm_stf_dft): the complex64 amplitude of the
    SU wavelet at path for frequency freq, float-identical to the
    reference's."""
    amp = np.zeros(2, np.float32)
    check(_lib.load().gm_stf_dft(str(path).encode(), physics, freq, ptr(amp)))
    return complex(np.complex64(amp[0] + 1j * amp[1]))
