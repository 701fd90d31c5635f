"""Drop-in: the reference's UNMODIFIED drivers forward_shot_AC
(src/AC/forward_shot_AC.c) and grad_obj_AC (src/AC/grad_obj_AC.c), built
from the reference tree against include/germaine_umfpack.h and linked with
libgermaine_umfpack.so (oracle/_ref/libgermaine_ref_dropin.so, made by
`make -C oracle dropin`), so that their UMFPACK calls factorise and solve
on the GPU.  Checked against the oracle: the same float arithmetic around
SuperLU FP64 solves of M = A^T.

Tolerances: seismograms are the reference's float casts of FP64 solutions
that agree to 1e-10, so they differ only where a rounding flips: 1e-6
relative.  The gradient and misfit are accumulated in float by the
reference over shots and frequencies; against the FP64 restatement they
agree to 1e-5 relative."""
import numpy as np
import pytest

import oracle as O
from oracle import sparse as OS
from tests.models import inclusion_ac, random_smooth
from tests.test_gpu_forward_grad import _observed, oracle_forward, oracle_grad

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.dropin_available(), reason="oracle/_ref/libgermaine_ref_dropin.so not built")]


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _case(seed=0):
    nx, ny, dh, npml = 72, 46, 10.0, 10
    vp, rho = inclusion_ac(nx, ny, dh, npml, radius=80.0)
    vp = vp * random_smooth(nx, ny, 0.9, 1.1, seed)
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    nx0 = nx - 2 * npml
    xs = np.linspace(2 * dh, (nx0 - 3) * dh, 4).astype(np.float32)
    ys = np.full(4, 3 * dh, np.float32)
    rx = np.arange(1, nx0 - 1, dtype=np.int32)
    ry = np.full(rx.size, 3, np.int32)
    return g, vp, rho, xs, ys, rx, ry


def test_reference_forward_shot_ac_on_gpu():
    g, vp, rho, xs, ys, rx, ry = _case()
    d = O.RefDropin(g)
    for freq in (8.0, 17.0):
        seis = d.forward_shot_ac(freq, vp, rho, xs, ys, rx, ry)
        X, _ = oracle_forward(g, O.PHYS_AC, vp, rho, [freq], xs, ys)
        idx = [OS.receiver_read_index(g, int(a), int(b)) for a, b in zip(rx, ry)]
        ref = OS.vec2mat(X[0].T)[:, idx]
        assert _rel(seis, ref) < 1e-6


@pytest.mark.parametrize("stf_inv", [0, 1], ids=["l2", "stf"])
def test_reference_grad_obj_ac_on_gpu(stf_inv):
    g, vp, rho, xs, ys, rx, ry = _case(seed=1)
    freqs = [7.0, 13.0]
    obs = _observed(g, O.PHYS_AC, vp, rho, freqs, xs, ys, rx, ry)
    d = O.RefDropin(g)
    grad, l2 = d.grad_obj_ac(freqs, vp, rho, xs, ys, rx, ry, obs, stf_inv=stf_inv)
    r0, _, rl2 = oracle_grad(g, O.PHYS_AC, vp, rho, freqs, xs, ys, rx, ry, obs, stf_inv, 1)
    assert _rel(grad.ravel(), r0) < 1e-5
    if stf_inv == 1:   # with STF_INV = 0 the reference's misfit accumulator is uninitialised
        assert abs(l2 - rl2) / rl2 < 1e-5


def test_reference_grad_obj_ac_rtm_on_gpu():
    """RTM_FD_AC's call of grad_obj_AC (INVMAT = 2, src/AC/RTM_FD_AC.c:190):
    the unmodified reference driver through the UMFPACK shim against the
    engine's own INVMAT = 2 path and the FP64 oracle."""
    from germaine_b200 import Engine
    g, vp, rho, xs, ys, rx, ry = _case(seed=2)
    freqs = [7.0, 13.0]
    obs = _observed(g, O.PHYS_AC, vp, rho, freqs, xs, ys, rx, ry)
    d = O.RefDropin(g)
    grad, l2 = d.grad_obj_ac(freqs, vp, rho, xs, ys, rx, ry, obs, stf_inv=1, invmat=2)
    d.lib.dropin_set_invmat(1)
    r0, _, rl2 = oracle_grad(g, O.PHYS_AC, vp, rho, freqs, xs, ys, rx, ry, obs, 1, 1, invmat=2)
    assert _rel(grad.ravel(), r0) < 1e-5
    assert abs(l2 - rl2) / rl2 < 1e-5
    with Engine(g.nx, g.ny, g.dh, g.npml) as e:
        e.set_model(vp, rho)
        e.factor(freqs)
        e.set_invmat(2)
        g0, _, _, _ = e.grad_obj(xs, ys, rx, ry, obs, stf_inv=1)
    assert _rel(g0, grad.ravel()) < 1e-5
