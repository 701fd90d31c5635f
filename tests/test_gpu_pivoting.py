"""Threshold partial pivoting inside the 32-pivot blocks of the upper
(blocked) levels.  UMFPACK, which the FP64 path replaces, pivots with a
relative tolerance of 0.1 by default; the engine does the same within each
32-pivot block of the fronts with more than 32 pivots (gm_config.pivot_tol).

The 3 Hz operator of the 841 x 227 benchmark grid (thrust model, 20-point
PML: well short of a wavelength at 3 Hz) has small pivots on those levels.
On the CPU, an LU in the engine's elimination order with diagonal pivots
only leaves a relative residual of 6.4e-11 (SuperLU with partial pivoting:
1.9e-14), and a multifrontal replay with exchanges inside the upper levels'
32-row blocks brings it to 5e-13 with 8 exchanges.  Here: the GPU
factorisation exchanges rows, its direct solve (before any refinement
sweep) is far more accurate than with static pivots only, and both
orientations (M x = b and M^T x = b, whose substitutions apply the
exchanges at different points) end at the residual target, checked on the
CPU against the assembled operator."""
import numpy as np
import pytest

import oracle as O
from oracle import sparse as OS
from germaine_b200 import GM_SYS_A, GM_SYS_AT, Engine
from germaine_b200.synthetic import thrust_model

pytestmark = pytest.mark.gpu

NX0, NY0, DH, NPML, FREQ = 801, 187, 25.0, 20, 3.0


def _first_residual(pivot_tol, sys, b, vp, rho):
    nx, ny = NX0 + 2 * NPML, NY0 + 2 * NPML
    with Engine(nx, ny, DH, NPML, pivot_tol=pivot_tol) as e:
        e.set_model(vp, rho)
        e.factor([FREQ])
        swaps = e.stats()["pivot_swaps"]
        x = e.solve(b, sys)
        first = e.refine_report()[0]["first_residual"]
        final = e.stats()["ir_residual"]
        trip = e.triplets(0)
    return swaps, first, final, x, trip


@pytest.mark.parametrize("sys", [GM_SYS_A, GM_SYS_AT])
def test_row_exchanges_restore_the_direct_solve_accuracy(sys):
    vp, rho = thrust_model(NX0, NY0, DH, NPML, seed=2024)
    nx, ny = NX0 + 2 * NPML, NY0 + 2 * NPML
    rng = np.random.default_rng(7)
    b = rng.standard_normal((nx * ny, 4)) + 1j * rng.standard_normal((nx * ny, 4))
    swaps, first, final, x, trip = _first_residual(0.0, sys, b, vp, rho)
    swaps0, first0, _, _, _ = _first_residual(-1.0, sys, b, vp, rho)
    assert swaps > 0 and swaps0 == 0
    assert first < 1e-11, first                  # the direct solve, before refinement
    assert first * 10 < first0, (first, first0)  # static pivots only: far less accurate
    assert final <= 1e-10
    g = O.Grid(nx=nx, ny=ny, dh=DH, npml=NPML)
    M = OS.operator(OS.assembled_matrix(g, *trip), 0)
    if sys == GM_SYS_AT:
        M = M.T
    r = b - M @ x
    rel = np.linalg.norm(r, axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 1e-10, rel
