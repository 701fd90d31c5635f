"""Parity at the benchmark configurations themselves, both precision paths,
against the FP64 oracle (the reference's assembly + SuperLU on the operator
UMFPACK factorises, M = A^T):

* C1 -- inclusion model, 201 x 101 interior at 10 m + 20-point PML
  (241 x 141), 15 Hz, 20 spikes on model row 3, 201 receivers on row 3;
* C2 -- seeded thrust model, 801 x 187 interior at 25 m + 20-point PML
  (841 x 227), the 2, 3 and 11 Hz matrices of the 2-11 Hz stage (the lowest,
  worst-conditioned ones and the highest), 100 shots on row 2, 800
  receivers.

The solve sites replaced are umfpack_zi_solve at src/AC/forward_shot_AC.c:88
(forward) and src/AC/grad_obj_AC.c:121,147 (forward and adjoint of the
gradient).  Tolerances: FP64 wavefields (the double solution vectors)
<= 1e-10 relative L2, mixed-precision ones <= 1e-8, float seismograms
<= 2e-6, FP64 gradient <= 1e-8 and mixed gradient <= 1e-6 relative to the
FP64 oracle gradient; every refined solve at residual <= 1e-10."""
import numpy as np
import pytest

import oracle as O
from oracle import sparse as OS
from germaine_b200 import GM_PHYS_AC, GM_PREC_C64_IR, GM_PREC_FP64, Engine
from germaine_b200.synthetic import inclusion_model, line_acquisition, thrust_model

pytestmark = pytest.mark.gpu

PRECISIONS = [(GM_PREC_FP64, 1e-10, 1e-8), (GM_PREC_C64_IR, 1e-8, 1e-6)]


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


class _Oracle:
    """SuperLU factors and forward solutions of one configuration."""

    def __init__(self, g, m0, m1, freqs, xs, ys, rx, ry):
        asm = O.Ref(g) if O.ref_available() else O.Port(g)
        self.g, self.freqs, self.xs, self.ys, self.rx, self.ry = g, freqs, xs, ys, rx, ry
        self.solvers, self.X = [], []
        for f in freqs:
            A = OS.assembled_matrix(g, *asm.assemble(GM_PHYS_AC, f, m0, m1))
            ds = OS.DirectSolver(OS.operator(A))
            self.solvers.append(ds)
            self.X.append(ds.solve(OS.spike_rhs(g, GM_PHYS_AC, f, xs, ys)))
        self.idx = [OS.receiver_read_index(g, int(a), int(b)) for a, b in zip(rx, ry)]
        self.seis = np.stack([OS.vec2mat(x.T)[:, self.idx] for x in self.X])

    def gradient(self, obs, m0, m1):
        """FP64 restatement of grad_obj_AC (misfit 1, no source estimate)."""
        g = self.g
        kadj = [OS.adjoint_index(g, int(a), int(b)) for a, b in zip(self.rx, self.ry)]
        dh2 = float(np.float32(g.dh) * np.float32(g.dh))
        Xa, stfu = [], np.ones((len(self.freqs), len(self.xs)), complex)
        for i, ds in enumerate(self.solvers):
            Badj = np.zeros((g.n, len(self.xs)), complex)
            for s in range(len(self.xs)):
                _, res, w = OS.residual_fp64(self.seis[i, s], obs[i, s], 0, 1)
                stfu[i, s] = w / abs(w)
                Badj[kadj, s] = np.conj(res) / dh2      # distinct receivers: assignment order is immaterial
            Xa.append(ds.solve(Badj))
        g0, _ = OS.gradient_fp64(g, GM_PHYS_AC, self.freqs, np.stack(self.X), np.stack(Xa), stfu, vp=m0, rho=m1)
        return g0


def _check_forward(e, orc, tol_x):
    ns = len(orc.xs)
    seis, _ = e.forward(orc.xs, orc.ys, orc.rx, orc.ry)
    st = e.stats()
    assert st["ir_residual"] <= 1e-10, f"refined residual {st['ir_residual']:.3e}"
    X = e.wavefield_fp64(0, ns)
    for i, f in enumerate(orc.freqs):
        err = _rel(X[i], orc.X[i])
        assert err <= tol_x, f"{f} Hz: wavefield differs from the oracle by {err:.3e}"
        assert _rel(seis[i], orc.seis[i]) <= 2e-6


# ---------------------------------------------------------------- C1
@pytest.fixture(scope="module")
def c1():
    nx0, ny0, dh, npml = 201, 101, 10.0, 20
    vp, rho = inclusion_model(nx0, ny0, dh, npml)
    g = O.Grid(nx=nx0 + 2 * npml, ny=ny0 + 2 * npml, dh=dh, npml=npml)
    xs = np.linspace(2 * dh, (nx0 - 3) * dh, 20).astype(np.float32)
    ys = np.full(20, 3 * dh, np.float32)
    rx = np.arange(1, nx0 + 1, dtype=np.int32)          # 201 receivers
    ry = np.full(rx.size, 3, np.int32)
    return g, vp, rho, _Oracle(g, vp, rho, [15.0], xs, ys, rx, ry)


@pytest.mark.parametrize("precision,tol_x,tol_g", PRECISIONS, ids=["fp64", "mixed"])
def test_c1_forward_matches_oracle(c1, precision, tol_x, tol_g):
    g, vp, rho, orc = c1
    assert g.nx * g.ny == 33_981
    with Engine(g.nx, g.ny, g.dh, g.npml, precision=precision) as e:
        e.set_model(vp, rho)
        e.factor(orc.freqs)
        assert e.stats()["nonzero"] == 303_541
        _check_forward(e, orc, tol_x)


# ---------------------------------------------------------------- C2
@pytest.fixture(scope="module")
def c2():
    nx0, ny0, dh, npml = 801, 187, 25.0, 20
    vp, rho = thrust_model(nx0, ny0, dh, npml, seed=2024)
    g = O.Grid(nx=nx0 + 2 * npml, ny=ny0 + 2 * npml, dh=dh, npml=npml)
    xs, ys, rx, ry = line_acquisition(nx0, dh, 100, 2)
    return g, vp, rho, _Oracle(g, vp, rho, [2.0, 3.0, 11.0], xs, ys, rx, ry)


@pytest.mark.parametrize("precision,tol_x,tol_g", PRECISIONS, ids=["fp64", "mixed"])
def test_c2_forward_matches_oracle(c2, precision, tol_x, tol_g):
    g, vp, rho, orc = c2
    assert g.nx * g.ny == 190_907 and len(orc.rx) == 800
    with Engine(g.nx, g.ny, g.dh, g.npml, precision=precision) as e:
        e.set_model(vp, rho)
        e.factor(orc.freqs)
        _check_forward(e, orc, tol_x)


@pytest.fixture(scope="module")
def c2_gradient(c2):
    g, vp, rho, orc = c2
    # observed data: the FP64 engine's seismograms of a 3 % smooth perturbation
    from tests.models import random_smooth
    vp_true = (vp * random_smooth(g.nx, g.ny, 0.97, 1.03, 17, corr=20.0)).astype(np.float32)
    with Engine(g.nx, g.ny, g.dh, g.npml) as e:
        e.set_model(vp_true, rho)
        e.factor(orc.freqs[1:])
        obs, _ = e.forward(orc.xs, orc.ys, orc.rx, orc.ry)
    sub = _Oracle.__new__(_Oracle)
    sub.__dict__.update(orc.__dict__)
    sub.freqs, sub.solvers, sub.X, sub.seis = orc.freqs[1:], orc.solvers[1:], orc.X[1:], orc.seis[1:]
    return sub, obs, sub.gradient(obs, vp, rho)


@pytest.mark.parametrize("precision,tol_x,tol_g", PRECISIONS, ids=["fp64", "mixed"])
def test_c2_gradient_matches_oracle(c2, c2_gradient, precision, tol_x, tol_g):
    """grad_obj over the 3 and 11 Hz matrices with 100 shots."""
    g, vp, rho, _ = c2
    orc, obs, g_ref = c2_gradient
    with Engine(g.nx, g.ny, g.dh, g.npml, precision=precision) as e:
        e.set_model(vp, rho)
        e.factor(orc.freqs)
        _, _, l2, _ = e.grad_obj(orc.xs, orc.ys, orc.rx, orc.ry, obs)
        assert e.stats()["ir_residual"] <= 1e-10
        g0, _ = e.gradient_fp64()
        xa = e.wavefield_fp64(1, len(orc.xs))
    assert np.isfinite(l2) and l2 > 0
    assert np.all(np.isfinite(xa))
    err = _rel(g0, g_ref)
    assert err <= tol_g, f"gradient differs from the FP64 oracle by {err:.3e}"
