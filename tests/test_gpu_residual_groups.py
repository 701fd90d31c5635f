"""The residual check (and the refinement's residual) covers every right-hand
side.  It runs full groups of 32 right-hand sides, one per lane, and the
last few (at most 8) in a segmented form whose lanes split the grid line
instead.  Here only those last right-hand sides are non-zero, so a form that
skipped them would report a zero residual (the zero columns have a zero
solution and a zero residual): with complex64 factors the direct solve must
report a first residual well above zero, the refinement (which forms r for
exactly those columns) must still reach the target, and the returned
solution must satisfy M x = b on the CPU.  nrhs = 1, 4, 7: only the
segmented form runs; 36, 100: a full group (or three) and a tail of 4."""
import numpy as np
import pytest

import oracle as O
from oracle import sparse as OS
from germaine_b200 import GM_PREC_C64_IR, GM_PREC_FP64, Engine
from tests.models import inclusion_ac, random_smooth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [GM_PREC_C64_IR, GM_PREC_FP64], ids=["c64ir", "fp64"])
@pytest.mark.parametrize("nrhs", [1, 4, 7, 36, 100])
def test_residual_check_sees_the_last_right_hand_sides(precision, nrhs):
    nx, ny, dh, npml = 71, 53, 10.0, 10
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    vp, rho = inclusion_ac(nx, ny, dh, npml)
    vp = vp * random_smooth(nx, ny, 0.85, 1.15, 5)
    rng = np.random.default_rng(nrhs)
    tail = nrhs % 32 if nrhs % 32 and nrhs % 32 <= 8 else nrhs
    b = np.zeros((g.n, nrhs), complex)
    b[:, nrhs - tail:] = rng.standard_normal((g.n, tail)) + 1j * rng.standard_normal((g.n, tail))
    with Engine(nx, ny, dh, npml, precision=precision, leaf_max=24) as e:
        e.set_model(vp, rho)
        e.factor([12.0])
        x = e.solve(b)
        rep = e.refine_report()[0]
        final = e.stats()["ir_residual"]
        trip = e.triplets(0)
    if precision == GM_PREC_C64_IR:
        assert 1e-9 < rep["first_residual"] < 1e-2, rep   # complex64 factors: visibly above zero
        assert rep["sweeps"] >= 1, rep
    else:
        assert 0 < rep["first_residual"] <= 1e-10, rep
    assert final <= 1e-10
    M = OS.operator(OS.assembled_matrix(g, *trip), 0)
    r = b - M @ x
    nb = np.linalg.norm(b, axis=0)
    live = nb > 0
    rel = np.linalg.norm(r[:, live], axis=0) / nb[live]
    assert rel.max() <= 1e-10, rel
    assert np.abs(x[:, ~live]).max(initial=0.0) == 0.0
