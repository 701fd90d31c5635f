"""Diagonal Hessians on the GPU (gm_hessian) and their application to the
gradient (gm_apply_hess).

* GM_HESS_SHIN = hessian_shin_AC / hessian_shin_TE
  (src/AC/hessian_shin_AC.c:48-141), GM_HESS_GREEN = hessian_AC /
  hessian_TE (src/AC/hessian_AC.c:48-174): against the FP64 restatement
  (oracle/sparse.py: hessian_fp64, every (shot, receiver) term formed on its
  own, SuperLU solves of M = A^T) to 1e-8 relative in FP64 and 2e-6 for the
  float output (the sum rounded to float, then frame-tapered in float as the
  reference does, so that frame points overflow to inf where the
  reference's do), and against the reference's own drivers run through the
  UMFPACK shim (oracle/_ref/libgermaine_ref_dropin.so).  The reference
  forms each term in complex float and sums in float, so there the bar is
  the float sum's rounding: 2e-5 relative.  The file the reference writes
  (<JACOBIAN>_hess) is gm_write_model's layout byte for byte.
* gm_apply_hess = apply_hess_AC (src/AC/apply_hess_AC.c:11-40):
  bit-identical to the reference's output in the committed fixture."""
import os

import numpy as np
import pytest

import oracle as O
from oracle import sparse as OS
from germaine_b200 import (GM_HESS_GREEN, GM_HESS_SHIN, GM_PHYS_AC, GM_PHYS_SH, GM_PHYS_TE, GM_PREC_C64_IR, Engine,
                           GmError, _lib, apply_hess, files)
from tests.test_gpu_forward_grad import _case
from tests.test_oracle_pin import _bits, hess_cases

pytestmark = pytest.mark.gpu

needs_dropin = pytest.mark.skipif(not O.dropin_available(), reason="oracle/_ref/libgermaine_ref_dropin.so not built")


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _rel_f32(h, r):
    """Relative error of a float output against a float reference, entries
    beyond the float range required to be inf on both sides (the TE epsilon
    Hessian, |Omega^2|^2 |F|^2, exceeds 3.4e38 at GPR frequencies; the
    reference holds it in float and stores inf there as well)."""
    h = np.asarray(h, np.float32).reshape(-1)
    r = np.asarray(r, np.float32).reshape(-1)
    assert np.array_equal(np.isinf(h), np.isinf(r))
    fin = np.isfinite(r)
    hf, rf = h[fin].astype(np.float64), r[fin].astype(np.float64)
    nr = np.linalg.norm(rf)
    return float(np.linalg.norm(hf - rf) / nr) if nr > 0 else float(np.max(np.abs(hf), initial=0.0))


def oracle_hessian(g, physics, mode, m0, m1, freqs, xs, ys, rx, ry):
    """FP64 Hessians (h0, h1) tapered, and the float outputs the reference's
    order gives (the sums rounded to float, then tapered in float)."""
    port = O.Port(g)
    src = OS.hessian_source_physics(physics, mode)
    X, solvers = [], []
    for f in freqs:
        ds = OS.DirectSolver(OS.operator(OS.assembled_matrix(g, *port.assemble(physics, f, m0, m1))))
        solvers.append(ds)
        X.append(ds.solve(OS.spike_rhs(g, src, f, xs, ys, port)))
    Xg = None
    if mode == GM_HESS_GREEN:
        B = OS.hess_green_rhs(g, physics, rx, ry)
        Xg = np.stack([s.solve(B) for s in solvers])   # UMFPACK_A for both physics
    u0, u1 = OS.hessian_fp64(g, physics, mode, freqs, np.stack(X), Xg, vp=m0, rho=m1, port=port, tapered=False)
    coef, passes = OS.grad_frame(g, port)
    fac = coef ** passes
    r0, r1 = u0 * fac, (u1 * fac if u1 is not None else None)
    f0 = OS.taper_float(g, u0, port)
    f1 = OS.taper_float(g, u1, port) if u1 is not None else None
    return r0, r1, f0, f1


def _engine_hessian(physics, mode, g, m0, m1, freqs, xs, ys, rx, ry, precision=None):
    kw = {} if precision is None else {"precision": precision}
    with Engine(g.nx, g.ny, g.dh, g.npml, physics=physics, leaf_max=32, **kw) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        h0, h1 = e.hessian(xs, ys, rx, ry, mode=mode)
        d0, d1 = e.hessian_fp64()
    return h0, h1, d0, d1


@pytest.mark.parametrize("mode", [GM_HESS_SHIN, GM_HESS_GREEN], ids=["shin", "green"])
@pytest.mark.parametrize("physics", [GM_PHYS_AC, GM_PHYS_TE], ids=["ac", "te"])
def test_hessian_matches_fp64_oracle(physics, mode):
    g, m0, m1, freqs, xs, ys, rx, ry = _case(physics, seed=3)
    h0, h1, d0, d1 = _engine_hessian(physics, mode, g, m0, m1, freqs, xs, ys, rx, ry)
    r0, r1, f0, f1 = oracle_hessian(g, physics, mode, m0, m1, freqs, xs, ys, rx, ry)
    assert _rel(d0, r0) < 1e-8 and _rel_f32(h0, f0) < 2e-6
    assert np.all(d0 >= 0)
    if physics == GM_PHYS_TE:
        assert _rel(d1, r1) < 1e-8 and _rel_f32(h1, f1) < 2e-6
    else:
        assert h1 is None


def test_hessian_mixed_precision_within_1e6():
    g, m0, m1, freqs, xs, ys, rx, ry = _case(GM_PHYS_AC, seed=4)
    _, _, d0, _ = _engine_hessian(GM_PHYS_AC, GM_HESS_GREEN, g, m0, m1, freqs, xs, ys, rx, ry,
                                  precision=GM_PREC_C64_IR)
    r0, *_ = oracle_hessian(g, GM_PHYS_AC, GM_HESS_GREEN, m0, m1, freqs, xs, ys, rx, ry)
    assert _rel(d0, r0) < 1e-6


@needs_dropin
@pytest.mark.parametrize("mode", [GM_HESS_SHIN, GM_HESS_GREEN], ids=["shin", "green"])
@pytest.mark.parametrize("physics", [GM_PHYS_AC, GM_PHYS_TE], ids=["ac", "te"])
def test_hessian_matches_reference_drivers(physics, mode, short_tmp):
    g, m0, m1, freqs, xs, ys, rx, ry = _case(physics, seed=5)
    if mode == GM_HESS_GREEN:
        rx, ry = rx[::3], ry[::3]    # the reference solves every receiver for every shot
    h0, h1, _, _ = _engine_hessian(physics, mode, g, m0, m1, freqs, xs, ys, rx, ry)
    jac = os.path.join(short_tmp, "jac")
    ref = O.RefDropin(g)
    r0, r1 = ref.hessian(physics, mode, freqs, m0, m1, xs, ys, rx, ry, jac)
    # the reference's sum_grad_MPI never fills grid point (NX, NY) (its
    # reduction starts one element early): compare every other point
    body = np.ones(g.n, bool)
    body[-1] = False
    assert _rel_f32(h0[body], r0.reshape(-1)[body]) < 2e-5
    suffix = ["_hess"] if physics == GM_PHYS_AC else ["_hess_sigma", "_hess_epsilon"]
    for name, arr in zip(suffix, (r0, r1)):
        ours = os.path.join(short_tmp, "ours")
        files.write_model(ours, arr)
        with open(jac + name, "rb") as a, open(ours, "rb") as b:
            assert a.read() == b.read()
    if physics == GM_PHYS_TE:
        assert _rel_f32(h1[body], r1.reshape(-1)[body]) < 2e-5


def test_hessian_errors():
    g, m0, m1, freqs, xs, ys, rx, ry = _case(GM_PHYS_AC)
    with Engine(g.nx, g.ny, g.dh, g.npml, leaf_max=32) as e:
        with pytest.raises(GmError):     # before any factorisation
            e.hessian(xs, ys)
        e.set_model(m0, m1)
        e.factor(freqs)
        with pytest.raises(GmError):     # Green's functions need receivers
            e.hessian(xs, ys, mode=GM_HESS_GREEN)
        with pytest.raises(GmError):
            e.hessian(xs, ys, rx, ry, mode=3)
        with pytest.raises(GmError):
            e.hessian_fp64()             # nothing computed yet
    gs, s0, s1, fs, *_ = _case(GM_PHYS_SH)
    with Engine(gs.nx, gs.ny, gs.dh, gs.npml, physics=GM_PHYS_SH, leaf_max=32) as e:
        e.set_model(s0, s1)
        e.factor(fs[:1])
        with pytest.raises(GmError):     # no SH Hessian in the reference
            e.hessian(xs[:1], ys[:1])


def test_apply_hess_matches_reference_fixture():
    for nx, ny, eps, grad, hess, ref, mx in hess_cases():
        out, m = apply_hess(grad, hess, eps)
        assert np.array_equal(_bits(out), _bits(ref)) and m == mx


def test_apply_hess_device_buffers():
    import torch
    nx, ny, eps, grad, hess, ref, mx = hess_cases()[0]
    dg = torch.from_numpy(grad.copy()).cuda()
    dh = torch.from_numpy(hess).cuda()
    lib = _lib.load()
    _lib.check(lib.gm_apply_hess(0, grad.size, eps, _lib.ptr(dg), _lib.ptr(dh), None))
    assert np.array_equal(_bits(dg.cpu().numpy()), _bits(ref))
    assert lib.gm_apply_hess(0, 0, eps, _lib.ptr(dg), _lib.ptr(dh), None) == _lib.GM_ERROR_INVALID
