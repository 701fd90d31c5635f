"""TEST ORACLE for the GERMAINE per-frequency hot path.

Test infrastructure only: tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py may import this
package, and only as the checker or the timed CPU baseline.  The product
(``germaine_b200``) never imports it.

Two CPU implementations live here:

* ``port``  -- liboracle_port.so, this project's plain-C restatement
  (oracle/port.c) of the reference's assembly, PML, source, receiver,
  residual and gradient arithmetic, bit-faithful in float/double;
* ``ref``   -- oracle/_ref/libgermaine_ref.so, the reference's own C sources
  compiled in place by oracle/Makefile (only where the reference tree is
  present; the built library travels with the repository snapshot);
* ``dropin`` -- oracle/_ref/libgermaine_ref_dropin.so, the reference's
  unmodified drivers forward_shot_AC / grad_obj_AC linked against the
  product's UMFPACK shim (libgermaine_umfpack.so): not a checker but the
  object under test of tests/test_gpu_dropin.py, run against the checkers
  above.

The sparse direct solve (UMFPACK in the reference, an un-vendored
SuiteSparse dependency with no pinned version) is restated with SciPy's
SuperLU in complex128 on the operator UMFPACK actually factorises
(oracle/sparse.py).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle_port.so")
REF_SO = os.path.join(HERE, "_ref", "libgermaine_ref.so")
DROPIN_SO = os.path.join(HERE, "_ref", "libgermaine_ref_dropin.so")

PHYS_AC, PHYS_SH, PHYS_TE = 1, 2, 4

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


@dataclass(frozen=True)
class Grid:
    """Full modelling grid INCLUDING the PML frame (NX, NY after
    forward_AC.c:44-45), spacing DH [m], PML width NPML, FREE_SURF, A0_PML
    and the Laplace damping S."""

    nx: int
    ny: int
    dh: float
    npml: int
    free_surf: int = 0
    a0_pml: float = 90.0
    s: float = 0.0

    @property
    def fsshift(self) -> int:
        return 0 if self.free_surf else self.npml

    @property
    def n(self) -> int:
        return self.nx * self.ny

    @property
    def nonzero(self) -> int:
        return 9 * self.nx * self.ny - 6 * self.nx - 6 * self.ny + 4


class _PortGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("npml", ctypes.c_int),
                ("free_surf", ctypes.c_int), ("fsshift", ctypes.c_int),
                ("dh", ctypes.c_float), ("a0_pml", ctypes.c_float), ("s", ctypes.c_float)]


def _pg(g: Grid) -> _PortGrid:
    return _PortGrid(g.nx, g.ny, g.npml, g.free_surf, g.fsshift, g.dh, g.a0_pml, g.s)


_port_lib = None
_ref_lib = None


def load_port():
    global _port_lib
    if _port_lib is None:
        if not os.path.exists(PORT_SO):
            raise RuntimeError(f"{PORT_SO} missing: run `make -C oracle port`")
        lib = ctypes.CDLL(PORT_SO)
        P = ctypes.POINTER(_PortGrid)
        lib.port_pml.argtypes = [P, ctypes.c_float, _f32p]
        lib.port_assemble.argtypes = [P, ctypes.c_int, ctypes.c_float, _f32p, _f32p, _f64p, _f64p, _i32p, _i32p]
        lib.port_assemble.restype = ctypes.c_int
        lib.port_rhs_source.argtypes = [P, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, _f64p, _f64p]
        lib.port_vec2mat.argtypes = [ctypes.c_int, _f64p, _f64p, _f32p, _f32p]
        lib.port_calc_seis.argtypes = [P, _f32p, _f32p, ctypes.c_int, _i32p, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p]
        lib.port_calc_res.argtypes = [_f32p, _f32p, _f32p, _f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p]
        lib.port_calc_res.restype = ctypes.c_float
        lib.port_rhs_adj.argtypes = [P, _f32p, _f32p, ctypes.c_int, _i32p, _i32p, _f64p, _f64p]
        lib.port_ass_grad_ac.argtypes = [P, ctypes.c_float, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p]
        lib.port_ass_grad_te.argtypes = [P, ctypes.c_float, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p]
        lib.port_grad_frame_coeff.argtypes = [P, _f32p]
        lib.port_cp_grad_frame.argtypes = [P, _f32p]
        lib.port_gradient_scalars.argtypes = [P, ctypes.c_int, ctypes.c_float, _f32p, _f32p]
        lib.port_gauss_filt.argtypes = [P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _f32p]
        lib.port_apply_hess.argtypes = [ctypes.c_int, ctypes.c_float, _f32p, _f32p]
        lib.port_apply_hess.restype = ctypes.c_float
        lib.port_lbfgs.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p,
                                   _f32p, _f32p, ctypes.c_void_p, ctypes.c_float, _f32p, _f32p, _f32p, _f32p, _f32p,
                                   _f32p]
        lib.port_lbfgs_rotate.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f32p]
        lib.port_check_descent.argtypes = [P, ctypes.c_int, _f32p, _f32p]
        lib.port_check_descent.restype = ctypes.c_float
        lib.port_precond_tapers.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, _f32p]
        lib.port_srt_field.argtypes = [P, ctypes.c_float, ctypes.c_float, ctypes.c_float, _f32p]
        lib.port_taper_grad_shot1.argtypes = [P, ctypes.c_int, ctypes.c_int, _f32p, _f32p, ctypes.c_int, _i32p, _i32p,
                                              _f32p]
        _port_lib = lib
    return _port_lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def load_ref():
    global _ref_lib
    if _ref_lib is None:
        if not ref_available():
            raise RuntimeError(f"{REF_SO} missing: run `make -C oracle ref` where the reference tree exists")
        lib = ctypes.CDLL(REF_SO)
        lib.ref_set_grid.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float]
        lib.ref_nonzero.restype = ctypes.c_int
        lib.ref_pml.argtypes = [ctypes.c_float, _f32p]
        lib.ref_assemble.argtypes = [ctypes.c_int, ctypes.c_float, _f32p, _f32p, _f64p, _f64p, _i32p, _i32p]
        lib.ref_assemble.restype = ctypes.c_int
        lib.ref_rhs_source.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, _f64p, _f64p]
        lib.ref_vec2mat.argtypes = [_f64p, _f64p, _f32p, _f32p]
        lib.ref_calc_seis.argtypes = [_f32p, _f32p, ctypes.c_int, _i32p, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p]
        lib.ref_calc_res.argtypes = [_f32p, _f32p, _f32p, _f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p]
        lib.ref_calc_res.restype = ctypes.c_float
        lib.ref_read_stf_dft.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_float, _f32p]
        lib.ref_rhs_adj.argtypes = [_f32p, _f32p, ctypes.c_int, _i32p, _i32p, _f64p, _f64p]
        lib.ref_ass_grad_ac.argtypes = [ctypes.c_float, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p]
        lib.ref_ass_grad_te.argtypes = [ctypes.c_float, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p]
        lib.ref_cp_grad_frame.argtypes = [_f32p]
        lib.ref_gauss_filt.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _f32p]
        cp, i = ctypes.c_char_p, ctypes.c_int
        lib.ref_write_seis.argtypes = [cp, i, i, i, i, _f32p, _f32p]
        lib.ref_read_seis.argtypes = [cp, i, i, i, i, _f32p, _f32p]
        lib.ref_writemod_true.argtypes = [cp, i, i, _f32p]
        lib.ref_writemod.argtypes = [cp, i, i, _f32p]
        lib.ref_readmod.argtypes = [cp, _f32p, _f32p]
        lib.ref_apply_hess.argtypes = [ctypes.c_float, _f32p, _f32p]
        lib.ref_taper_grad_shot.argtypes = [ctypes.c_float, ctypes.c_int, _f32p, _f32p, ctypes.c_int, _i32p, _i32p,
                                            ctypes.c_int, _f32p]
        lib.ref_taper_grad_shot1.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f32p, ctypes.c_int, _i32p, _i32p,
                                             _f32p]
        f_ = ctypes.c_float
        lib.ref_tikhonov_cost_te.restype = f_
        lib.ref_tikhonov_cost_te.argtypes = [ctypes.c_int, ctypes.c_int, f_, f_, f_, f_, f_, f_, _f32p, _f32p, f_]
        lib.ref_tikhonov_grad_te.argtypes = [ctypes.c_int, ctypes.c_int, f_, f_, f_, f_, f_, f_, _f32p, _f32p, _f32p,
                                             _f32p]
        lib.ref_apply_hess.restype = ctypes.c_float
        fp = _f32p
        lib.ref_lbfgs_ac.argtypes = [i, i, i, fp, fp, fp, fp, fp, fp, fp, fp, fp, fp, cp, fp]
        lib.ref_lbfgs_te.argtypes = [i, i, i, i, ctypes.c_float, ctypes.c_float, ctypes.c_float, fp, fp, fp, fp, fp, fp,
                                     fp, fp, fp, fp, fp, fp, fp, fp, fp, cp, fp, fp]
        lib.ref_lbfgs_rotate.argtypes = [i, i, fp, fp]
        lib.ref_dotp_matrix.argtypes = [fp, fp]
        lib.ref_dotp_matrix.restype = ctypes.c_float
        lib.ref_precond.argtypes = [cp, i, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, i, i, i, fp]
        lib.ref_precond.restype = ctypes.c_int
        _ref_lib = lib
    return _ref_lib


# the reference formats file names into char[STRING_SIZE] buffers (include/fd.h:27)
REF_STRING_SIZE = 74


def _ref_name(path, longest_suffix: str) -> bytes:
    """A path the reference will extend by at most longest_suffix; refuses
    names that would overflow its fixed file-name buffers."""
    b = os.fsencode(path)
    if len(b) + len(longest_suffix) + 1 > REF_STRING_SIZE:
        raise ValueError(f"{path!r}{longest_suffix} does not fit the reference's {REF_STRING_SIZE}-byte file names")
    return b


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# --------------------------------------------------------------- port API
class Port:
    """Restated hot-path arithmetic (oracle/port.c) on flat row-major
    [NY][NX] arrays (grid point (i, j), 1-based, is index (j-1)*NX+(i-1))."""

    def __init__(self, g: Grid):
        self.g = g
        self.lib = load_port()
        self._pg = _pg(g)

    def pml(self, freq: float) -> np.ndarray:
        out = np.zeros(4 * (self.g.nx + 2) + 4 * (self.g.ny + 2), np.float32)
        self.lib.port_pml(ctypes.byref(self._pg), freq, out)
        return out

    def assemble(self, physics: int, freq: float, m0, m1):
        nz = self.g.nonzero
        ar = np.zeros(nz); ai = np.zeros(nz)
        ir = np.zeros(nz, np.int32); ic = np.zeros(nz, np.int32)
        c = self.lib.port_assemble(ctypes.byref(self._pg), physics, freq, _f32(m0).ravel(), _f32(m1).ravel(), ar, ai, ir, ic)
        if c != nz:
            raise RuntimeError(f"port_assemble wrote {c} triplets, expected {nz}")
        return ar, ai, ir, ic

    def rhs_source(self, physics, freq, xsrc, ysrc):
        rr = np.zeros(self.g.n); ri = np.zeros(self.g.n)
        self.lib.port_rhs_source(ctypes.byref(self._pg), physics, freq, xsrc, ysrc, rr, ri)
        return rr, ri

    def vec2mat(self, x: np.ndarray):
        n = self.g.n
        xr = np.zeros(n + 1); xi = np.zeros(n + 1)
        xr[:n] = x.real; xi[:n] = x.imag
        pr = np.zeros(n, np.float32); pi = np.zeros(n, np.float32)
        self.lib.port_vec2mat(n, xr, xi, pr, pi)
        return pr, pi

    def calc_seis(self, pr, pi, recx, recy, ishot, nshots, nfreq, sr, si):
        self.lib.port_calc_seis(ctypes.byref(self._pg), _f32(pr), _f32(pi), len(recx),
                                np.asarray(recx, np.int32), np.asarray(recy, np.int32),
                                ishot, nshots, nfreq, sr, si)

    def calc_res(self, calr, cali, obsr, obsi, stf_inv=0, invmat=1, misfit=1):
        ntr = len(calr)
        rr = np.zeros(ntr, np.float32); ri = np.zeros(ntr, np.float32); stf = np.zeros(2, np.float32)
        l2 = self.lib.port_calc_res(_f32(calr), _f32(cali), _f32(obsr), _f32(obsi), ntr, stf_inv, invmat, misfit, rr, ri, stf)
        return float(l2), rr, ri, stf

    def rhs_adj(self, resr, resi, recx, recy):
        rr = np.zeros(self.g.n); ri = np.zeros(self.g.n)
        self.lib.port_rhs_adj(ctypes.byref(self._pg), _f32(resr), _f32(resi), len(recx),
                              np.asarray(recx, np.int32), np.asarray(recy, np.int32), rr, ri)
        return rr, ri

    def ass_grad_ac(self, freq, stf, fr, fi, lr, li, vp, rho, grad):
        self.lib.port_ass_grad_ac(ctypes.byref(self._pg), freq, _f32(stf), _f32(fr), _f32(fi),
                                  _f32(lr), _f32(li), _f32(vp), _f32(rho), grad)

    def ass_grad_te(self, freq, stf, fr, fi, lr, li, gsig, geps):
        self.lib.port_ass_grad_te(ctypes.byref(self._pg), freq, _f32(stf), _f32(fr), _f32(fi),
                                  _f32(lr), _f32(li), gsig, geps)

    def grad_frame_coeff(self):
        c = np.zeros(self.g.n, np.float32)
        self.lib.port_grad_frame_coeff(ctypes.byref(self._pg), c)
        return c

    def cp_grad_frame(self, grad):
        self.lib.port_cp_grad_frame(ctypes.byref(self._pg), grad)

    def srt_field(self, xc, yc, radius):
        """Radial taper coefficients of one centre (metres), [NY*NX] float."""
        c = np.zeros(self.g.n, np.float32)
        self.lib.port_srt_field(ctypes.byref(self._pg), xc, yc, radius, c)
        return c

    def taper_grad_shot(self, grad, radius, sx, sy, rx, ry, ishot):
        """taper_grad_shot on a [NY*NX] float gradient: the source of shot
        ishot (0-based), then each receiver, one float product each."""
        out = _f32(grad).copy()
        out *= self.srt_field(float(sx[ishot]), float(sy[ishot]), radius)
        for x, y in zip(rx, ry):
            out *= self.srt_field(np.float32(x) * np.float32(self.g.dh), np.float32(y) * np.float32(self.g.dh), radius)
        return out

    def taper_grad_shot1(self, grad, filtsize, sx, sy, rx, ry):
        out = _f32(grad).copy()
        self.lib.port_taper_grad_shot1(ctypes.byref(self._pg), filtsize, len(sx), _f32(sx), _f32(sy), len(rx),
                                       np.asarray(rx, np.int32), np.asarray(ry, np.int32), out)
        return out

    def gauss_filt(self, grad, vref, fc_low, fsg, fsg1):
        """Filtered copy of a [NY][NX] gradient (gauss_filt)."""
        out = np.ascontiguousarray(grad, np.float32).copy()
        self.lib.port_gauss_filt(ctypes.byref(self._pg), vref, fc_low, fsg, fsg1, out.reshape(-1))
        return out

    # ---- file formats (numpy restatement) ----
    def seis_bytes(self, seis, keep_last=False):
        """write_seis_AC (src/AC/write_seis_AC.c:53-67): (re, im) float pairs,
        frequency outer, shot, receiver inner.  Its gather
        (src/AC/write_seis_AC.c:43-44) reduces the 1-based arrays from
        element 0, so element n never arrives and the last sample is 0."""
        s = np.array(seis, np.complex64).reshape(-1)
        if not keep_last:
            s[-1] = 0
        return s.tobytes()

    def model_true_bytes(self, grid, idx=1, idy=1):
        """writemod_true (src/writemod_true.c:26-34): interior columns, x outer."""
        g, fs = self.g, self.g.fsshift
        inner = np.asarray(grid, np.float32)[fs:g.ny - g.npml, g.npml:g.nx - g.npml]
        return np.ascontiguousarray(inner[::idy, ::idx].T).tobytes()

    def model_bytes(self, grid, idx=1, idy=1):
        """writemod format 3 (src/writemod.c:24-30): full grid, x outer."""
        return np.ascontiguousarray(np.asarray(grid, np.float32)[::idy, ::idx].T).tobytes()

    def model_from_bytes(self, data):
        """readmod (src/readmod.c:43-104): interior read x outer, then the
        frame filled with the nearest interior value."""
        g, fs = self.g, self.g.fsshift
        nx0, ny0 = g.nx - 2 * g.npml, g.ny - g.npml - fs
        inner = np.frombuffer(data, np.float32, nx0 * ny0).reshape(nx0, ny0).T
        return np.pad(inner, ((fs, g.npml), (g.npml, g.npml)), mode="edge")

    def apply_hess(self, grad, hess, eps_hess):
        """apply_hess_AC: (preconditioned copy of grad, MAX_HESS)."""
        out = np.ascontiguousarray(grad, np.float32).copy()
        mx = self.lib.port_apply_hess(out.size, eps_hess, out.reshape(-1), _f32(hess).reshape(-1))
        return out, float(mx)

    def precond(self, grad, spatfilter=0, vref=0.0, fc_low=1.0, fsg=0.0, fsg1=0.0, taper_hor=0, gradt2=0,
                taper=None):
        """precond (src/precond.c:10-24): gauss_filt, taper_grad_hor, taper_grad_file."""
        out = np.ascontiguousarray(grad, np.float32).copy()
        if spatfilter == 1:
            out = self.gauss_filt(out, vref, fc_low, fsg, fsg1)
        tp = _f32(taper).ravel() if taper is not None else None
        self.lib.port_precond_tapers(ctypes.byref(self._pg), taper_hor, gradt2,
                                     None if tp is None else tp.ctypes.data_as(ctypes.c_void_p), out.reshape(-1))
        return out

    def gradient_scalars(self, physics, freq):
        """(Omega^2, Omega) of ass_grad_AC / ass_grad_TE as complex64 values."""
        a = np.zeros(2, np.float32); b = np.zeros(2, np.float32)
        self.lib.port_gradient_scalars(ctypes.byref(self._pg), physics, freq, a, b)
        return complex(a[0], a[1]), complex(b[0], b[1])


class Ref:
    """The reference's own sources (compiled into oracle/_ref); same call
    shapes as :class:`Port`.  Holds process-global reference state, so only
    one grid is active at a time."""

    def __init__(self, g: Grid):
        self.g = g
        self.lib = load_ref()
        self.lib.ref_set_grid(g.nx, g.ny, g.dh, g.npml, g.free_surf, g.a0_pml, g.s)

    def nonzero(self):
        return self.lib.ref_nonzero()

    def pml(self, freq):
        out = np.zeros(4 * (self.g.nx + 2) + 4 * (self.g.ny + 2), np.float32)
        self.lib.ref_pml(freq, out)
        return out

    def assemble(self, physics, freq, m0, m1):
        nz = self.g.nonzero
        ar = np.zeros(nz); ai = np.zeros(nz)
        ir = np.zeros(nz, np.int32); ic = np.zeros(nz, np.int32)
        if self.lib.ref_assemble(physics, freq, _f32(m0).ravel(), _f32(m1).ravel(), ar, ai, ir, ic) != 0:
            raise RuntimeError("ref_assemble failed")
        return ar, ai, ir, ic

    def rhs_source(self, physics, freq, xsrc, ysrc):
        rr = np.zeros(self.g.n); ri = np.zeros(self.g.n)
        self.lib.ref_rhs_source(physics, freq, xsrc, ysrc, rr, ri)
        return rr, ri

    def vec2mat(self, x):
        n = self.g.n
        xr = np.zeros(n + 1); xi = np.zeros(n + 1)
        xr[:n] = x.real; xi[:n] = x.imag
        pr = np.zeros(n, np.float32); pi = np.zeros(n, np.float32)
        self.lib.ref_vec2mat(xr, xi, pr, pi)
        return pr, pi

    def calc_seis(self, pr, pi, recx, recy, ishot, nshots, nfreq, sr, si, nf):
        self.lib.ref_calc_seis(_f32(pr), _f32(pi), len(recx), np.asarray(recx, np.int32),
                               np.asarray(recy, np.int32), ishot, nshots, nf, nfreq, sr, si)

    def calc_res(self, calr, cali, obsr, obsi, stf_inv=0, invmat=1, misfit=1):
        ntr = len(calr)
        rr = np.zeros(ntr, np.float32); ri = np.zeros(ntr, np.float32); stf = np.zeros(2, np.float32)
        l2 = self.lib.ref_calc_res(_f32(calr), _f32(cali), _f32(obsr), _f32(obsi), ntr, 1, 1, 1, 1,
                                   stf_inv, invmat, misfit, rr, ri, stf)
        return float(l2), rr, ri, stf

    def rhs_adj(self, resr, resi, recx, recy):
        rr = np.zeros(self.g.n); ri = np.zeros(self.g.n)
        self.lib.ref_rhs_adj(_f32(resr), _f32(resi), len(recx), np.asarray(recx, np.int32),
                             np.asarray(recy, np.int32), rr, ri)
        return rr, ri

    def ass_grad_ac(self, freq, stf, fr, fi, lr, li, vp, rho, grad):
        self.lib.ref_ass_grad_ac(freq, _f32(stf), _f32(fr), _f32(fi), _f32(lr), _f32(li), _f32(vp), _f32(rho), grad)

    def ass_grad_te(self, freq, stf, fr, fi, lr, li, gsig, geps):
        self.lib.ref_ass_grad_te(freq, _f32(stf), _f32(fr), _f32(fi), _f32(lr), _f32(li), gsig, geps)

    def cp_grad_frame(self, grad):
        self.lib.ref_cp_grad_frame(grad)

    def taper_grad_shot(self, grad, radius, sx, sy, rx, ry, ishot):
        out = _f32(grad).copy()
        self.lib.ref_taper_grad_shot(radius, len(sx), _f32(sx), _f32(sy), len(rx), np.asarray(rx, np.int32),
                                     np.asarray(ry, np.int32), ishot, out)
        return out

    def tikhonov_cost_te(self, sigma, epsilon, l2, norm1, norm2, beta1, beta2, lambda1, lambda2, idx=1, idy=1):
        return float(self.lib.ref_tikhonov_cost_te(idx, idy, norm1, norm2, beta1, beta2, lambda1, lambda2,
                                                   _f32(sigma).ravel(), _f32(epsilon).ravel(), l2))

    def tikhonov_grad_te(self, gsig, geps, sigma, epsilon, norm1, norm2, beta1, beta2, lambda1, lambda2, idx=1,
                         idy=1):
        gs = _f32(gsig).ravel().copy()
        ge = _f32(geps).ravel().copy()
        self.lib.ref_tikhonov_grad_te(idx, idy, norm1, norm2, beta1, beta2, lambda1, lambda2, _f32(sigma).ravel(),
                                      _f32(epsilon).ravel(), gs, ge)
        return gs, ge

    def taper_grad_shot1(self, grad, filtsize, sx, sy, rx, ry):
        out = _f32(grad).copy()
        self.lib.ref_taper_grad_shot1(filtsize, len(sx), _f32(sx), _f32(sy), len(rx), np.asarray(rx, np.int32),
                                      np.asarray(ry, np.int32), out)
        return out

    def gauss_filt(self, grad, vref, fc_low, fsg, fsg1):
        out = np.ascontiguousarray(grad, np.float32).copy()
        self.lib.ref_gauss_filt(vref, fc_low, fsg, fsg1, out.reshape(-1))
        return out

    def apply_hess(self, grad, hess, eps_hess):
        """apply_hess_AC: (preconditioned copy of grad, MAX_HESS)."""
        out = np.ascontiguousarray(grad, np.float32).copy()
        mx = self.lib.ref_apply_hess(eps_hess, out.reshape(-1), _f32(hess).reshape(-1))
        return out, float(mx)

    def precond(self, workdir, grad, spatfilter=0, vref=0.0, fc_low=1.0, fsg=0.0, fsg1=0.0, taper_hor=0, gradt2=0,
                taper=None):
        """The reference's precond; `taper` (NX0*NY0, x outer) is written to
        <workdir>/taper.bin, where taper_grad_file reads it."""
        if taper is not None:
            _f32(taper).ravel().tofile(os.path.join(workdir, "taper.bin"))
        out = np.ascontiguousarray(grad, np.float32).copy()
        rc = self.lib.ref_precond(os.fsencode(workdir), spatfilter, vref, fc_low, fsg, fsg1, taper_hor, gradt2,
                                  int(taper is not None), out.reshape(-1))
        if rc != 0:
            raise RuntimeError("ref_precond: could not enter " + str(workdir))
        return out

    # ---- file formats: the reference writes / reads the files itself ----
    def write_seis(self, prefix, stage, seis):
        """write_seis_AC: <prefix>_p_stage_<stage>.bin from complex [nf][nshots][ntr]."""
        nf, ns, ntr = seis.shape
        self.lib.ref_write_seis(_ref_name(prefix, f"_p_stage_{stage}.bin"), stage, nf, ns, ntr, _f32(seis.real).ravel(),
                                _f32(seis.imag).ravel())

    def read_seis(self, prefix, stage, nf, nshots, ntr):
        """read_seis_AC of <prefix>_p_stage_<stage>.bin."""
        re = np.zeros(nf * nshots * ntr, np.float32); im = np.zeros_like(re)
        self.lib.ref_read_seis(_ref_name(prefix, f"_p_stage_{stage}.bin"), stage, nf, nshots, ntr, re, im)
        return (re + 1j * im).astype(np.complex64).reshape(nf, nshots, ntr)

    def writemod_true(self, path, grid, idx=1, idy=1):
        self.lib.ref_writemod_true(_ref_name(path, ""), idx, idy, _f32(grid).ravel())

    def writemod(self, path, grid, idx=1, idy=1):
        self.lib.ref_writemod(_ref_name(path, ""), idx, idy, _f32(grid).ravel())

    def readmod(self, mfile):
        """readmod of <mfile>.vp / <mfile>.rho -> (vp, rho) [NY][NX] with the frame."""
        vp = np.zeros(self.g.n, np.float32); rho = np.zeros_like(vp)
        self.lib.ref_readmod(_ref_name(mfile, ".germaine.rho"), vp, rho)
        return vp.reshape(self.g.ny, self.g.nx), rho.reshape(self.g.ny, self.g.nx)


def dropin_available() -> bool:
    return os.path.exists(DROPIN_SO)


class RefDropin:
    """The reference's own drivers running their UMFPACK calls on the GPU
    (oracle/ref_dropin.c).  Holds process-global reference state."""

    def __init__(self, g: Grid):
        if not dropin_available():
            raise RuntimeError(f"{DROPIN_SO} missing: run `make -C oracle dropin` where the reference tree exists")
        self.g = g
        lib = ctypes.CDLL(DROPIN_SO)
        lib.ref_set_grid.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_float, ctypes.c_float]
        lib.dropin_forward_shot_ac.argtypes = [ctypes.c_float, _f32p, _f32p, ctypes.c_int, _f32p, _f32p, ctypes.c_int,
                                               _i32p, _i32p, _f32p, _f32p]
        lib.dropin_grad_obj_ac.argtypes = [ctypes.c_int, _f32p, _f32p, _f32p, ctypes.c_int, _f32p, _f32p, ctypes.c_int,
                                           _i32p, _i32p, _f32p, _f32p, ctypes.c_int, ctypes.c_int, _f32p]
        lib.dropin_grad_obj_ac.restype = ctypes.c_float
        lib.dropin_set_invmat.argtypes = [ctypes.c_int]
        cp, i = ctypes.c_char_p, ctypes.c_int
        lib.dropin_hessian_ac.argtypes = [i, i, _f32p, _f32p, _f32p, i, _f32p, _f32p, i, _i32p, _i32p, cp, _f32p]
        lib.dropin_hessian_te.argtypes = [i, i, _f32p, _f32p, _f32p, i, _f32p, _f32p, i, _i32p, _i32p, cp, _f32p,
                                          _f32p]
        self.lib = lib
        lib.ref_set_grid(g.nx, g.ny, g.dh, g.npml, g.free_surf, g.a0_pml, g.s)

    def forward_shot_ac(self, freq, vp, rho, xs, ys, rx, ry):
        """Seismograms [nshots][ntr] complex64 of forward_shot_AC."""
        ns, ntr = len(xs), len(rx)
        sr = np.zeros(ns * ntr, np.float32); si = np.zeros(ns * ntr, np.float32)
        self.lib.dropin_forward_shot_ac(freq, _f32(vp).ravel(), _f32(rho).ravel(), ns, _f32(xs), _f32(ys), ntr,
                                        np.ascontiguousarray(rx, np.int32), np.ascontiguousarray(ry, np.int32), sr, si)
        return (sr + 1j * si).reshape(ns, ntr).astype(np.complex64)

    def grad_obj_ac(self, freqs, vp, rho, xs, ys, rx, ry, obs, stf_inv=0, misfit=1, invmat=1):
        """(gradient [NY][NX] float32, L2) of grad_obj_AC over one stage."""
        nf, ns, ntr = len(freqs), len(xs), len(rx)
        obs = np.asarray(obs, np.complex64).reshape(nf, ns, ntr)
        grad = np.zeros(self.g.n, np.float32)
        self.lib.dropin_set_invmat(invmat)
        l2 = self.lib.dropin_grad_obj_ac(nf, _f32(freqs), _f32(vp).ravel(), _f32(rho).ravel(), ns, _f32(xs),
                                         _f32(ys), ntr, np.ascontiguousarray(rx, np.int32),
                                         np.ascontiguousarray(ry, np.int32), _f32(obs.real).ravel(),
                                         _f32(obs.imag).ravel(), stf_inv, misfit, grad)
        return grad.reshape(self.g.ny, self.g.nx), float(l2)

    def hessian(self, physics, mode, freqs, m0, m1, xs, ys, rx, ry, jacobian):
        """hessian_shin_{AC,TE} (mode 2) or hessian_{AC,TE} (mode 1) over one
        stage: (hess0, hess1) [NY][NX] float32 (AC: hess, None; TE: sigma,
        epsilon with MAT1_NORM = MAT2_NORM = 1).  The drivers write their
        <jacobian>_hess* files too."""
        nf, ns, ntr = len(freqs), len(xs), len(rx)
        args = (mode, nf, _f32(freqs), _f32(m0).ravel(), _f32(m1).ravel(), ns, _f32(xs), _f32(ys), ntr,
                np.ascontiguousarray(rx, np.int32), np.ascontiguousarray(ry, np.int32),
                _ref_name(jacobian, "_hess_epsilon"))
        h0 = np.zeros(self.g.n, np.float32)
        shape = (self.g.ny, self.g.nx)
        if physics == PHYS_TE:
            h1 = np.zeros(self.g.n, np.float32)
            self.lib.dropin_hessian_te(*args, h0, h1)
            return h0.reshape(shape), h1.reshape(shape)
        self.lib.dropin_hessian_ac(*args, h0)
        return h0.reshape(shape), None


class PortLbfgs:
    """The restated l-BFGS (port.c: port_lbfgs) with its state: history y, s
    ([m][nvec]) and the previous gradient / model, as the reference keeps
    them in its LBFGS vectors and "*.old" files."""

    def __init__(self, g: Grid, m: int, nclass: int = 1):
        self.g, self.m, self.nclass = g, m, nclass
        self.lib = load_port()
        self._pg = _pg(g)
        self.nvec = nclass * g.n
        self.y = np.zeros(m * self.nvec, np.float32)
        self.s = np.zeros(m * self.nvec, np.float32)
        self.old_grad = np.zeros(self.nvec, np.float32)
        self.old_model = np.zeros(self.nvec, np.float32)
        self.q = np.zeros(self.nvec, np.float32)
        self.r = np.zeros(self.nvec, np.float32)
        self.scal = np.zeros(2 * m + 1, np.float32)

    def step(self, first, pointer, grad, gradm, model, hess=None, eps_hess=0.0):
        out = np.zeros(self.nvec, np.float32)
        hs = _f32(hess).ravel() if hess is not None else None
        self.lib.port_lbfgs(ctypes.byref(self._pg), self.nclass, self.m, pointer, int(bool(first)), self.y, self.s,
                            _f32(grad).ravel(), _f32(gradm).ravel(), _f32(model).ravel(),
                            None if hs is None else hs.ctypes.data_as(ctypes.c_void_p), eps_hess, self.old_grad,
                            self.old_model, self.q, self.r, self.scal, out)
        return out.reshape(np.shape(gradm))

    def rotate(self):
        self.lib.port_lbfgs_rotate(self.m, self.nvec, self.y, self.s)

    def zero(self):
        self.y[:] = 0
        self.s[:] = 0

    def check_descent(self, hgrad, grad):
        p = float(self.lib.port_check_descent(ctypes.byref(self._pg), self.nclass, _f32(hgrad).ravel(),
                                              _f32(grad).ravel()))
        if p < 0.0:
            self.zero()
        return p


class RefLbfgs:
    """The reference's LBFGS / LBFGS_TE (oracle/_ref) with the persistent
    arrays the reference's FWI loop owns; it reads and writes its "*.old"
    files under `jacobian` (keep that path short: the reference formats file
    names into fixed buffers)."""

    def __init__(self, g: Grid, m: int, nclass: int, jacobian: str):
        self.g, self.m, self.nclass = g, m, nclass
        self.lib = load_ref()
        self.lib.ref_set_grid(g.nx, g.ny, g.dh, g.npml, g.free_surf, g.a0_pml, g.s)
        self.jac = _ref_name(jacobian, "_p_epsilon_grad.old")
        self.nvec = nclass * g.n
        self.y = np.zeros(m * self.nvec, np.float32)
        self.s = np.zeros(m * self.nvec, np.float32)
        self.rho = np.zeros(m, np.float32)
        self.alpha = np.zeros(m, np.float32)
        self.beta = np.zeros(m, np.float32)
        self.q = np.zeros(self.nvec, np.float32)
        self.r = np.zeros(self.nvec, np.float32)

    def step_ac(self, iter_, pointer, grad, gradm, vp):
        out = np.zeros(self.g.n, np.float32)
        self.lib.ref_lbfgs_ac(iter_, pointer, self.m, self.y, self.s, self.rho, self.alpha, self.q, self.r,
                              self.beta, _f32(grad).ravel(), _f32(gradm).ravel(), _f32(vp).ravel(), self.jac, out)
        return out.reshape(self.g.ny, self.g.nx)

    def step_te(self, reset, pointer, grad, gradm, model, norms, hess=None, eps_hess=0.0):
        """grad, gradm, model, hess: [2][NY][NX] (sigma, epsilon); model is
        sigma, epsilon before normalisation; norms = (MAT1_NORM, MAT2_NORM)."""
        n = self.g.n
        gs, ge = (_f32(a).ravel() for a in grad)
        ms, me = (_f32(a).ravel() for a in gradm)
        sg, ep = (_f32(a).ravel() for a in model)
        hs, he = ((_f32(a).ravel() for a in hess) if hess is not None else (np.zeros(n, np.float32),) * 2)
        o0 = np.zeros(n, np.float32); o1 = np.zeros(n, np.float32)
        self.lib.ref_lbfgs_te(int(bool(reset)), pointer, self.m, int(hess is not None), eps_hess, norms[0], norms[1],
                              self.y, self.s, self.rho, self.alpha, self.q, self.r, self.beta, gs, ge, ms, me, sg, ep,
                              hs, he, self.jac, o0, o1)
        return np.stack([o0, o1]).reshape(2, self.g.ny, self.g.nx)

    def rotate(self):
        self.lib.ref_lbfgs_rotate(self.m, self.nvec, self.y, self.s)


def ref_stf_dft(path: str, physics: int, freq: float) -> complex:
    """The reference's read_stf_dft (oracle/_ref) on the SU file at path:
    the complex64 amplitude at freq."""
    import numpy as np
    lib = load_ref()
    amp = np.zeros(2, np.float32)
    lib.ref_read_stf_dft(str(path).encode(), physics, freq, amp)
    return complex(np.complex64(amp[0] + 1j * amp[1]))
