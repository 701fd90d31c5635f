"""Trial models of a line search in one batch (gm_set_models,
gm_factor_models, gm_obj_each): the reference's obj_AC
(src/AC/obj_AC.c:10-145) re-assembles and re-factorises every trial model
of parabolicls_AC / wolfels_AC one after the other; here the (model,
frequency) pairs are factorised and solved together, and each matrix's
misfit equals the one-model-at-a-time result and the FP64 oracle's."""
import numpy as np
import pytest

from germaine_b200 import Engine, GmError
from tests.models import inclusion_ac, random_smooth
from tests.test_gpu_forward_grad import _observed, oracle_grad
import oracle as O

pytestmark = pytest.mark.gpu


def _case():
    nx, ny, dh, npml = 64, 44, 10.0, 10
    vp, rho = inclusion_ac(nx, ny, dh, npml, radius=60.0)
    vp = vp * random_smooth(nx, ny, 0.9, 1.1, 6)
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    nx0 = nx - 2 * npml
    xs = np.linspace(2 * dh, (nx0 - 3) * dh, 4).astype(np.float32)
    ys = np.full(4, 3 * dh, np.float32)
    rx = np.arange(1, nx0 - 1, dtype=np.int32)
    ry = np.full(rx.size, 3, np.int32)
    return g, vp, rho, xs, ys, rx, ry


def test_trial_models_batched_equal_one_at_a_time():
    g, vp, rho, xs, ys, rx, ry = _case()
    freqs = [7.0, 13.0]
    obs = _observed(g, 1, vp, rho, freqs, xs, ys, rx, ry)
    direction = random_smooth(g.nx, g.ny, -1.0, 1.0, 9)
    steps = [0.0, 0.02, 0.05]
    trials = np.stack([(vp * (1 + a * direction)).astype(np.float32) for a in steps])
    rhos = np.stack([rho] * len(steps))
    pairs = [(m, f) for m in range(len(steps)) for f in freqs]
    with Engine(g.nx, g.ny, g.dh, g.npml, leaf_max=32) as e:
        e.set_models(trials, rhos)
        e.factor_models([f for _, f in pairs], [m for m, _ in pairs])
        batch_obs = np.stack([obs[freqs.index(f)] for _, f in pairs])
        each = e.obj_each(xs, ys, rx, ry, batch_obs)
        seis_b, _ = e.forward(xs, ys, rx, ry)
        with pytest.raises(GmError):   # one gradient needs one model
            e.grad_obj(xs, ys, rx, ry, batch_obs)
    per_model = each.reshape(len(steps), len(freqs)).sum(axis=1)
    for m, a in enumerate(steps):
        with Engine(g.nx, g.ny, g.dh, g.npml, leaf_max=32) as e:
            e.set_model(trials[m], rho)
            e.factor(freqs)
            l2 = e.obj(xs, ys, rx, ry, obs)
            seis, _ = e.forward(xs, ys, rx, ry)
        assert abs(per_model[m] - l2) <= 2e-6 * abs(l2)
        for k in range(len(freqs)):
            sb = seis_b[m * len(freqs) + k]
            assert np.linalg.norm(sb - seis[k]) <= 2e-6 * np.linalg.norm(seis[k])
        _, _, rl2 = oracle_grad(g, 1, trials[m], rho, freqs, xs, ys, rx, ry, obs, 0, 1)
        assert abs(per_model[m] - rl2) <= 2e-6 * abs(rl2)


def test_model_index_checked():
    g, vp, rho, *_ = _case()
    with Engine(g.nx, g.ny, g.dh, g.npml, leaf_max=32) as e:
        e.set_models(np.stack([vp, vp]), np.stack([rho, rho]))
        with pytest.raises(GmError):
            e.factor_models([7.0, 9.0], [0, 2])
