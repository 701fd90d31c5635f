"""FWI on the engine (the C4 configuration and a small case):

* the exact discrete gradient (GM_OP_EXACT: residuals not zeroed, adjoint
  solve with M^T, the stencil's mass spread differentiated, no vec2mat shift)
  against central finite differences of the FP64 misfit on random interior
  cells;
* the reference's host loop fwi_FD_AC (src/AC/fwi_FD_AC.c:229-409:
  grad_obj_AC, device l-BFGS, parabolic line search, calc_mat_change_wolfe)
  over the engine, on the 801 x 187 thrust model from a 500 m Gaussian-
  smoothed start, 5 stages of 3 frequencies in 2-10 Hz, 100 shots, 801
  receivers: the misfit falls in every stage and the model moves towards the
  true one."""
import numpy as np
import pytest

from germaine_b200 import GM_OP_EXACT, Engine
from germaine_b200.engine import Lbfgs
from germaine_b200.fwi import FwiLog, FwiParams, run_stage
from germaine_b200.synthetic import line_acquisition, thrust_model
from tests.models import inclusion_ac, random_smooth

pytestmark = pytest.mark.gpu


def _misfits_of_models(e, vp_list, rho, freqs, xs, ys, rx, ry, obs):
    """FP64 misfit of each model over the frequencies (one batched
    factorisation of every (model, frequency) pair)."""
    nm, nf = len(vp_list), len(freqs)
    e.set_models(np.stack(vp_list), np.stack([rho] * nm))
    e.factor_models(np.tile(np.asarray(freqs, np.float32), nm), np.repeat(np.arange(nm, dtype=np.int32), nf))
    e.obj_each(xs, ys, rx, ry, np.tile(obs, (nm, 1, 1)))
    _, each = e.misfit_fp64()
    return each.reshape(nm, nf).sum(axis=1)


def _fd_check(e, vp, rho, freqs, xs, ys, rx, ry, obs, cells, rel_step, batch):
    e.set_model(vp, rho)
    e.factor(freqs)
    e.grad_obj(xs, ys, rx, ry, obs)
    g, _ = e.gradient_fp64()
    g = g.reshape(vp.shape)
    fd = []
    for i0 in range(0, len(cells), batch):
        models = []
        for (y, x) in cells[i0:i0 + batch]:
            h = rel_step * vp[y, x]
            for sgn in (1.0, -1.0):
                m = vp.copy()
                m[y, x] = np.float32(vp[y, x] + sgn * h)
                models.append(m)
        J = _misfits_of_models(e, models, rho, freqs, xs, ys, rx, ry, obs)
        for k, (y, x) in enumerate(cells[i0:i0 + batch]):
            hp = float(np.float32(vp[y, x] + rel_step * vp[y, x])) - float(vp[y, x])
            hm = float(vp[y, x]) - float(np.float32(vp[y, x] - rel_step * vp[y, x]))
            fd.append((J[2 * k] - J[2 * k + 1]) / (hp + hm))
    an = np.array([g[y, x] for (y, x) in cells])
    return an, np.array(fd)


def _cells(rng, nx, ny, npml, count):
    ys = rng.integers(npml + 2, ny - npml - 2, count)
    xs = rng.integers(npml + 2, nx - npml - 2, count)
    return list(zip(ys.tolist(), xs.tolist()))


def test_exact_gradient_matches_finite_differences_small():
    nx, ny, dh, npml = 64, 44, 10.0, 10
    vp, rho = inclusion_ac(nx, ny, dh, npml, radius=60.0)
    vp = (vp * random_smooth(nx, ny, 0.9, 1.1, 3)).astype(np.float32)
    nx0 = nx - 2 * npml
    xs = np.linspace(2 * dh, (nx0 - 3) * dh, 4).astype(np.float32)
    ys = np.full(4, 3 * dh, np.float32)
    rx = np.arange(1, nx0 - 1, dtype=np.int32)
    ry = np.full(rx.size, 3, np.int32)
    freqs = [9.0, 17.0]
    vtrue = (vp * random_smooth(nx, ny, 0.95, 1.05, 8)).astype(np.float32)
    with Engine(nx, ny, dh, npml, op_mode=GM_OP_EXACT, leaf_max=24) as e:
        e.set_model(vtrue, rho)
        e.factor(freqs)
        obs, _ = e.forward(xs, ys, rx, ry)
        cells = _cells(np.random.default_rng(1), nx, ny, npml, 12)
        an, fd = _fd_check(e, vp, rho, freqs, xs, ys, rx, ry, obs, cells, 1e-2, 6)
    # the assembly forms every coefficient in complex float (as the
    # reference does), so a relative step h perturbs the operator with
    # rounding noise of about 6e-8 / h; with h = 1e-2 that and the O(h^2)
    # error of the central difference stay below 1e-3
    assert np.linalg.norm(an - fd) / np.linalg.norm(fd) < 1e-3, (an, fd)


@pytest.fixture(scope="module")
def c4():
    nx0, ny0, dh, npml = 801, 187, 25.0, 20
    vtrue, rho = thrust_model(nx0, ny0, dh, npml, seed=2024)
    from scipy.ndimage import gaussian_filter
    vstart = gaussian_filter(vtrue.astype(np.float64), 500.0 / dh, mode="nearest").astype(np.float32)
    xs, ys, _, _ = line_acquisition(nx0, dh, 100, 2)
    rx = np.arange(1, nx0 + 1, dtype=np.int32)          # 801 receivers
    ry = np.full(rx.size, 2, np.int32)
    stages = [list(map(float, f)) for f in np.linspace(2.0, 10.0, 15).reshape(5, 3).astype(np.float32)]
    return nx0 + 2 * npml, ny0 + 2 * npml, dh, npml, vtrue, vstart, rho, xs, ys, rx, ry, stages


def test_c4_exact_gradient_finite_differences(c4):
    """Central differences on 50 random interior cells (at least NPML + 2
    from the edges) of the first stage's misfit, at the starting model."""
    nx, ny, dh, npml, vtrue, vstart, rho, xs, ys, rx, ry, stages = c4
    with Engine(nx, ny, dh, npml, op_mode=GM_OP_EXACT) as e:
        e.set_model(vtrue, rho)
        e.factor(stages[0])
        obs, _ = e.forward(xs, ys, rx, ry)
        cells = _cells(np.random.default_rng(4), nx, ny, npml, 50)
        an, fd = _fd_check(e, vstart, rho, stages[0], xs, ys, rx, ry, obs, cells, 1e-2, 5)
    assert np.linalg.norm(an - fd) / np.linalg.norm(fd) < 1e-3


def test_c4_fwi_stages_reduce_misfit(c4):
    nx, ny, dh, npml, vtrue, vstart, rho, xs, ys, rx, ry, stages = c4
    p = FwiParams(itermax=10, nlbfgs=10, eps_scale=0.01, scalefac=2.0, stepmax=6, pro=0.0,
                  vp_low=1500.0, vp_up=7000.0)
    log = FwiLog()
    vp = vstart.copy()
    interior = (slice(npml, ny - npml), slice(npml, nx - npml))
    err0 = np.linalg.norm((vstart - vtrue)[interior]) / np.linalg.norm(vtrue[interior])
    with Engine(nx, ny, dh, npml) as e, Lbfgs(nx, ny, npml, p.nlbfgs) as lb:
        for si, freqs in enumerate(stages, start=1):
            e.set_model(vtrue, rho)
            e.factor(freqs)
            obs, _ = e.forward(xs, ys, rx, ry)
            vp = run_stage(e, lb, vp, rho, freqs, xs, ys, rx, ry, obs, p, log, stage=si)
            e.set_model(vp, rho)
            e.factor(freqs)
            e.obj(xs, ys, rx, ry, obs)
            final, _ = e.misfit_fp64()
            first = log.misfit[log.stage.index(si)]
            assert final < first, f"stage {si}: misfit {first:.4e} -> {final:.4e}"
    err1 = np.linalg.norm((vp - vtrue)[interior]) / np.linalg.norm(vtrue[interior])
    assert len(log.misfit) >= 10
    assert err1 < err0, f"model error {err0:.4f} -> {err1:.4f}"
