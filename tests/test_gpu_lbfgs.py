"""The reference's l-BFGS update on the GPU (gm_lbfgs_*, gm_mat_change)
against the C restatement (oracle/port.c: port_lbfgs, itself pinned
bit-for-bit to the reference's LBFGS / LBFGS_TE in test_oracle_pin.py):
every search direction of a multi-iteration sequence is bit-identical,
including the history rotation, the TE two-class layout with and without
the diagonal-Hessian scaling, the loss-of-descent reset and a resume from
the previous gradient and model ("*.old" state)."""
import numpy as np
import pytest

import oracle as O
from germaine_b200 import GmError, Lbfgs, mat_change
from tests import lbfgs_cases as LC
from tests.test_oracle_pin import _bits

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(_bits(np.asarray(a, np.float32)), _bits(np.asarray(b, np.float32)))


@pytest.mark.parametrize("nx,ny,npml,m,iters", [(37, 29, 5, 3, 6), (841, 227, 20, 5, 8)], ids=["small", "thrust"])
def test_lbfgs_ac_bit_identical(nx, ny, npml, m, iters):
    g = LC.grid(nx, ny, npml)
    seq = LC.sequence(g, 1, iters, seed=3)
    port = O.PortLbfgs(g, m, 1)
    a = LC.run(lambda f, p, it, gr, gm, md, h: port.step(f, p, gr, gm, md), port.rotate, m, seq)
    with Lbfgs(nx, ny, npml, m) as d:
        b = LC.run(lambda f, p, it, gr, gm, md, h: d.step(f, p, gr, gm, md), d.rotate, m, seq)
        og, om = d.get_old()
    for x, y in zip(a, b):
        assert _same(x, y)
    assert _same(og.ravel(), seq[-1][0].ravel()) and _same(om.ravel(), seq[-1][2].ravel())


@pytest.mark.parametrize("with_hess", [False, True], ids=["gamma", "hessian"])
def test_lbfgs_te_bit_identical(with_hess):
    g, m, norms, eps = LC.grid(free_surf=1), 2, (0.01, 8.85e-11), 0.005
    seq = LC.sequence(g, 2, 5, seed=4)
    hs = (lambda h: h) if with_hess else (lambda h: None)
    port = O.PortLbfgs(g, m, 2)
    a = LC.run(lambda f, p, it, gr, gm, md, h: port.step(f, p, gr, gm, LC.normalise(md, norms), hs(h), eps),
               port.rotate, m, seq)
    with Lbfgs(g.nx, g.ny, g.npml, m, nclass=2, free_surf=1) as d:
        b = LC.run(lambda f, p, it, gr, gm, md, h: d.step(f, p, gr, gm, LC.normalise(md, norms), hs(h), eps),
                   d.rotate, m, seq)
    for x, y in zip(a, b):
        assert _same(x, y)


def test_check_descent_and_reset():
    g, m = LC.grid(), 2
    seq = LC.sequence(g, 1, 3, seed=5)
    port = O.PortLbfgs(g, m, 1)
    with Lbfgs(g.nx, g.ny, g.npml, m) as d:
        for k, (gr, gm, md, _) in enumerate(seq[:2]):
            hp = port.step(k == 0, 1, gr, gm, md)
            hd = d.step(k == 0, 1, gr, gm, md)
        assert _same(hp, hd)
        gr = seq[1][0]
        for direction in (hd, -hd):      # one of the two is not a descent direction
            pp = port.check_descent(direction, gr)
            pd = d.check_descent(direction, gr)
            assert _same(pp, pd)
        # after the reset (p < 0 for one of them) both histories are empty again
        gr, gm, md, _ = seq[2]
        assert _same(port.step(False, 2, gr, gm, md), d.step(False, 2, gr, gm, md))


def test_resume_from_previous_state():
    """A new engine given the previous gradient and model (the "*.old"
    files) continues exactly like the reference after a restart."""
    g, m = LC.grid(), 3
    seq = LC.sequence(g, 1, 2, seed=6)
    (g0, gm0, m0, _), (g1, gm1, m1, _) = seq
    port = O.PortLbfgs(g, m, 1)
    port.step(True, 1, g0, gm0, m0)
    want = port.step(False, 1, g1, gm1, m1)
    with Lbfgs(g.nx, g.ny, g.npml, m) as d:
        with pytest.raises(GmError):     # no previous state yet
            d.step(False, 1, g1, gm1, m1)
        d.set_old(g0, m0)
        assert _same(d.step(False, 1, g1, gm1, m1), want)
        with pytest.raises(GmError):
            d.step(False, m + 1, g1, gm1, m1)


@pytest.mark.parametrize("mode", [0, 1])
def test_mat_change_bit_identical(mode):
    rng = np.random.default_rng(7)
    old = rng.uniform(1500, 4500, 5000).astype(np.float32)
    h = (rng.standard_normal(5000) * 500).astype(np.float32)
    eps, low, up = np.float32(0.7), np.float32(1400.0), np.float32(4700.0)
    got = mat_change(h, old, eps, low, up, mode)
    v = (old + eps * h).astype(np.float32)
    if mode == 0:    # calc_mat_change_wolfe: outside the bounds keeps the old value
        want = np.where((v < low) | (v > up) | (v < 0), old, v)
    else:            # calc_mat_change_wolfe_multi_para: clamped
        want = np.clip(v, low, up)
    assert _same(got, want)
    assert np.any(got != v)              # the constraint was exercised
