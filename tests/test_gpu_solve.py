"""Multifrontal factor + multi-RHS solve on the GPU vs SuperLU (FP64) on the
operator UMFPACK factorises (M = A^T, or A in EXACT mode)."""
import numpy as np
import pytest

import oracle as O
from oracle import sparse as OS
from germaine_b200 import (GM_OP_EXACT, GM_OP_REF, GM_PHYS_AC, GM_PHYS_TE, GM_PREC_C64_IR, GM_PREC_FP64, GM_SYS_A,
                           GM_SYS_AT, Engine)
from germaine_b200._lib import GM_REFINE_MODE_AUTO, GM_REFINE_MODE_GMRES, GM_REFINE_MODE_IR
from tests.models import inclusion_ac, random_smooth, te_model

pytestmark = pytest.mark.gpu


def _setup(nx, ny, dh, npml, physics=GM_PHYS_AC, seed=0):
    if physics == GM_PHYS_TE:
        return te_model(nx, ny, seed)
    vp, rho = inclusion_ac(nx, ny, dh, npml)
    return vp * random_smooth(nx, ny, 0.85, 1.15, seed), rho


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("precision", [GM_PREC_FP64, GM_PREC_C64_IR], ids=["fp64", "c64ir"])
@pytest.mark.parametrize("op_mode", [GM_OP_REF, GM_OP_EXACT], ids=["ref", "exact"])
@pytest.mark.parametrize("sys_", [GM_SYS_A, GM_SYS_AT], ids=["A", "At"])
def test_solve_matches_superlu(precision, op_mode, sys_):
    nx, ny, dh, npml = 71, 53, 10.0, 10
    freqs = [12.0, 25.0]
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    m0, m1 = _setup(nx, ny, dh, npml, seed=3)
    rng = np.random.default_rng(11)
    nrhs = 13
    b = rng.standard_normal((len(freqs), g.n, nrhs)) + 1j * rng.standard_normal((len(freqs), g.n, nrhs))
    with Engine(nx, ny, dh, npml, precision=precision, op_mode=op_mode, leaf_max=24) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        x = e.solve(b, sys=sys_)
        st = e.stats()
    port = O.Port(g)
    for i, f in enumerate(freqs):
        A = OS.assembled_matrix(g, *port.assemble(1, f, m0, m1))
        ds = OS.DirectSolver(OS.operator(A, op_mode))
        xr = ds.solve(b[i], trans=(sys_ == GM_SYS_AT))
        err = _rel(x[i], xr)
        Mop = ds.M.T if sys_ == GM_SYS_AT else ds.M
        res = max(np.linalg.norm(Mop @ x[i][:, k] - b[i][:, k]) / np.linalg.norm(b[i][:, k]) for k in range(nrhs))
        assert res <= 1e-10, f"relative residual {res:.3e} (freq {f})"
        tol = 1e-10 if precision == GM_PREC_FP64 else 1e-8
        assert err <= tol, f"relative L2 error vs SuperLU {err:.3e} (freq {f})"
    assert st["ir_residual"] <= 1e-10


@pytest.mark.parametrize("shape", [(5, 5, 1), (9, 4, 1), (60, 9, 2), (13, 77, 3), (128, 31, 5)])
def test_solve_grid_shapes(shape):
    """Tiny, skinny and tall grids (ND leaves, single-front trees, uneven cuts)."""
    nx, ny, npml = shape
    dh = 20.0
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    m0, m1 = random_smooth(nx, ny, 1500.0, 3500.0, 5), random_smooth(nx, ny, 1000.0, 2500.0, 6)
    rng = np.random.default_rng(1)
    b = rng.standard_normal((1, g.n, 3)) + 1j * rng.standard_normal((1, g.n, 3))
    with Engine(nx, ny, dh, npml, leaf_max=16) as e:
        e.set_model(m0, m1)
        e.factor([7.0])
        x = e.solve(b)
    A = OS.assembled_matrix(g, *O.Port(g).assemble(1, 7.0, m0, m1))
    xr = OS.DirectSolver(OS.operator(A)).solve(b[0])
    assert _rel(x[0], xr) <= 1e-10


def test_te_transpose_solve():
    nx, ny, dh, npml = 48, 40, 0.025, 8
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    m0, m1 = _setup(nx, ny, dh, npml, physics=GM_PHYS_TE, seed=2)
    rng = np.random.default_rng(4)
    b = rng.standard_normal((1, g.n, 4)) + 1j * rng.standard_normal((1, g.n, 4))
    with Engine(nx, ny, dh, npml, physics=GM_PHYS_TE, leaf_max=32) as e:
        e.set_model(m0, m1)
        e.factor([2e8])
        x = e.solve(b, sys=GM_SYS_AT)
    A = OS.assembled_matrix(g, *O.Port(g).assemble(4, 2e8, m0, m1))
    xr = OS.DirectSolver(OS.operator(A)).solve(b[0], trans=True)
    assert _rel(x[0], xr) <= 1e-10


@pytest.mark.parametrize("precision,tc", [(GM_PREC_FP64, 0), (GM_PREC_C64_IR, 0), (GM_PREC_C64_IR, 96)],
                         ids=["fp64", "c64ir", "c64ir-tcgen05"])
def test_solve_large_fronts(precision, tc):
    """A grid whose upper fronts have contribution blocks above 96 rows; with
    tc_min_block = 96 the complex64 factorisation routes those blocks'
    updates to the tcgen05 kernel (counted in the statistics)."""
    nx, ny, dh, npml = 230, 170, 10.0, 12
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    m0, m1 = _setup(nx, ny, dh, npml, seed=8)
    rng = np.random.default_rng(12)
    b = rng.standard_normal((1, g.n, 6)) + 1j * rng.standard_normal((1, g.n, 6))
    with Engine(nx, ny, dh, npml, precision=precision, tc_min_block=tc) as e:
        e.set_model(m0, m1)
        e.factor([18.0])
        x = e.solve(b)
        st = e.stats()
    assert (st["tc_tiles"] > 0) == (tc > 0)
    A = OS.assembled_matrix(g, *O.Port(g).assemble(1, 18.0, m0, m1))
    ds = OS.DirectSolver(OS.operator(A))
    xr = ds.solve(b[0])
    assert st["max_front"] > 200
    res = max(np.linalg.norm(ds.M @ x[0][:, k] - b[0][:, k]) / np.linalg.norm(b[0][:, k]) for k in range(6))
    assert res <= 1e-10
    assert _rel(x[0], xr) <= (1e-10 if precision == GM_PREC_FP64 else 1e-8)
    if precision == GM_PREC_C64_IR:
        assert st["ir_iterations"] <= 4


def test_fp64_refinement_sweeps():
    """FP64 factors pass the first residual check, which therefore forms only
    the norms; a target below FP64 rounding forces sweeps, which must form
    the residual again and keep the solution at the SuperLU reference."""
    nx, ny, dh, npml = 40, 30, 10.0, 6
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    m0, m1 = random_smooth(nx, ny, 1500.0, 3500.0, 7), random_smooth(nx, ny, 1000.0, 2500.0, 8)
    rng = np.random.default_rng(9)
    b = rng.standard_normal((1, g.n, 5)) + 1j * rng.standard_normal((1, g.n, 5))
    with Engine(nx, ny, dh, npml, leaf_max=16, ir_tol=1e-30, ir_max_iter=2) as e:
        e.set_model(m0, m1)
        e.factor([9.0])
        x = e.solve(b)
        st = e.stats()
    assert st["ir_iterations"] == 2 and st["n_subst"] == 3
    assert st["ir_residual"] <= 1e-12
    A = OS.assembled_matrix(g, *O.Port(g).assemble(1, 9.0, m0, m1))
    xr = OS.DirectSolver(OS.operator(A)).solve(b[0])
    assert _rel(x[0], xr) <= 1e-10


@pytest.mark.parametrize("refine", [GM_REFINE_MODE_AUTO, GM_REFINE_MODE_IR, GM_REFINE_MODE_GMRES],
                         ids=["auto", "ir", "gmres"])
@pytest.mark.parametrize("sys_", [GM_SYS_A, GM_SYS_AT], ids=["A", "At"])
def test_mixed_refinement_modes(refine, sys_):
    """complex64 factors refined by plain sweeps, by GMRES-IR (FP64 Arnoldi,
    complex64 factors as right preconditioner) or by the automatic choice;
    every mode reaches the target and the SuperLU solution, and the
    per-matrix report names the method and its sweeps."""
    nx, ny, dh, npml = 90, 64, 10.0, 10
    freqs = [3.0, 11.0, 24.0]
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    m0, m1 = _setup(nx, ny, dh, npml, seed=21)
    rng = np.random.default_rng(5)
    nrhs = 37
    b = rng.standard_normal((len(freqs), g.n, nrhs)) + 1j * rng.standard_normal((len(freqs), g.n, nrhs))
    with Engine(nx, ny, dh, npml, precision=GM_PREC_C64_IR, leaf_max=24, refine=refine, gmres_restart=4) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        x = e.solve(b, sys=sys_)
        st = e.stats()
        rep = e.refine_report()
    assert st["ir_residual"] <= 1e-10
    assert len(rep) == len(freqs)
    port = O.Port(g)
    for i, f in enumerate(freqs):
        A = OS.assembled_matrix(g, *port.assemble(1, f, m0, m1))
        ds = OS.DirectSolver(OS.operator(A))
        xr = ds.solve(b[i], trans=(sys_ == GM_SYS_AT))
        assert _rel(x[i], xr) <= 1e-8
        r = rep[i]
        assert r["final_residual"] <= 1e-10 < r["first_residual"]
        assert r["sweeps"] >= 1
        if refine == GM_REFINE_MODE_IR:
            assert r["method"] == "ir"
        if refine == GM_REFINE_MODE_GMRES:
            assert r["method"] == "gmres"


@pytest.mark.parametrize("precision", [GM_PREC_FP64, GM_PREC_C64_IR], ids=["fp64", "c64ir"])
def test_autotuned_tiles_keep_the_solution(precision):
    """The autotuner picks, per level and pass, a candidate substitution
    tile where it beats the built-in one (the table names the resolved
    choice either way); solves with the tuned table give the SuperLU
    solution, and other right-hand-side counts keep the defaults."""
    nx, ny, dh, npml = 90, 64, 10.0, 10
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    m0, m1 = _setup(nx, ny, dh, npml, seed=13)
    rng = np.random.default_rng(2)
    nrhs = 45
    b = rng.standard_normal((2, g.n, nrhs)) + 1j * rng.standard_normal((2, g.n, nrhs))
    with Engine(nx, ny, dh, npml, precision=precision, leaf_max=24) as e:
        e.set_model(m0, m1)
        e.factor([8.0, 19.0])
        table = e.autotune(nrhs)
        assert len(table) == e.stats()["nlevels"]
        for fr, fs, br, bs in table:
            assert fr in (32, 64) and br in (32, 64) and fs in (32, 40) and bs in (32, 40)
        x = e.solve(b)
        x7 = e.solve(b[:, :, :7])
        assert e.stats()["ir_residual"] <= 1e-10
    port = O.Port(g)
    for i, f in enumerate([8.0, 19.0]):
        ds = OS.DirectSolver(OS.operator(OS.assembled_matrix(g, *port.assemble(1, f, m0, m1))))
        tol = 1e-10 if precision == GM_PREC_FP64 else 1e-8
        assert _rel(x[i], ds.solve(b[i])) <= tol
        assert _rel(x7[i], ds.solve(b[i][:, :7])) <= tol
