"""The batched multi-grid configuration (C3): 32 frequencies in 2-17 Hz,
each on its own grid at 5 points per minimum wavelength (400 x 100 to
1600 x 400 cells + PML, 9.4 M unknowns in all), 200 shots per frequency as
one right-hand-side block, complex64 factors with FP64 refinement, all grids
concurrently (one engine and stream per grid).  Every grid must meet the
residual target; a small grid and a large one are checked against the FP64
engine."""
import numpy as np
import pytest

from germaine_b200 import GM_PREC_C64_IR, GM_PREC_FP64, Engine
from germaine_b200.multigrid import c3_cases, run_multigrid, smooth_random_model

pytestmark = pytest.mark.gpu


def test_c3_all_grids_concurrently():
    cases = c3_cases()
    assert len(cases) == 32
    assert cases[0].shape == (140, 440) and cases[-1].shape == (440, 1640)
    rate, wall, recs = run_multigrid(cases, nshots=200, precision=GM_PREC_C64_IR, workers=32)
    assert len(recs) == 32 and rate > 0
    for r in recs:
        assert r["ir_residual"] <= 1e-10, r
        assert r["status"] >= 0
    print(f"C3: {rate:.0f} shot-solves/s, {wall * 1e3:.1f} ms for 32 grids x 200 shots")


@pytest.mark.parametrize("which", [0, 31], ids=["smallest", "largest"])
def test_c3_grid_mixed_matches_fp64(which):
    cases = c3_cases()
    c = cases[which]
    ny, nx = c.shape
    extent_x = max(q.nx0 * q.dh for q in cases)
    extent_y = max(q.ny0 * q.dh for q in cases)
    vp, rho = smooth_random_model(extent_x, extent_y, c.dh, c.nx0, c.ny0, c.npml, 7)
    xs = np.linspace(2 * c.dh, (c.nx0 - 3) * c.dh, 24).astype(np.float32)
    ys = np.full(xs.size, 2 * c.dh, np.float32)
    rx = np.arange(1, c.nx0, 4, dtype=np.int32)
    ry = np.full(rx.size, 2, np.int32)
    x = {}
    for prec in (GM_PREC_FP64, GM_PREC_C64_IR):
        with Engine(nx, ny, c.dh, c.npml, precision=prec) as e:
            e.set_model(vp, rho)
            e.factor([c.freq])
            e.forward(xs, ys, rx, ry)
            assert e.stats()["ir_residual"] <= 1e-10
            x[prec] = e.wavefield_fp64(0, xs.size)
    err = np.linalg.norm(x[GM_PREC_C64_IR] - x[GM_PREC_FP64]) / np.linalg.norm(x[GM_PREC_FP64])
    assert err < 1e-8
