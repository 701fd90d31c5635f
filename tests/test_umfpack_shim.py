"""UMFPACK-API shim (libgermaine_umfpack.so, include/germaine_umfpack.h):
the six calls of the reference's drivers, in the drivers' own sequence
(src/AC/forward_shot_AC.c:41-120), checked against SciPy (triplet
conversion) and against SuperLU FP64 solves of the matrix UMFPACK would
factorise (the solves, on the GPU)."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from oracle import sparse as OS
from germaine_b200 import _lib
from tests.models import inclusion_ac, random_smooth

P = _lib.ptr
vp_t = ctypes.c_void_p


def umf():
    return _lib.load_umfpack()


def triplet_to_col(n_row, n_col, ti, tj, tx=None, tz=None, want_map=False, packed=False):
    ti = np.ascontiguousarray(ti, np.int32)
    tj = np.ascontiguousarray(tj, np.int32)
    nz = ti.size
    ap = np.zeros(n_col + 1, np.int32)
    ai = np.zeros(max(nz, 1), np.int32)
    ax = az = None
    if tx is not None:
        ax = np.zeros(2 * max(nz, 1) if packed else max(nz, 1))
        if not packed:
            az = np.zeros(max(nz, 1))
    mp = np.zeros(max(nz, 1), np.int32) if want_map else None
    rc = umf().umfpack_zi_triplet_to_col(n_row, n_col, nz, P(ti), P(tj), P(tx), P(tz), P(ap), P(ai), P(ax), P(az),
                                         P(mp))
    return rc, ap, ai, ax, az, mp


def reference_flow_matrix(nx, ny, dh, npml, freq, seed):
    """Triplets of the reference's assembly (restated C, bit-identical to the
    reference) and the CSC arrays the driver hands UMFPACK: structure from
    triplet_to_col, values overwritten in triplet order
    (src/AC/forward_shot_AC.c:41-48)."""
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    vp, rho = inclusion_ac(nx, ny, dh, npml)
    vp = vp * random_smooth(nx, ny, 0.9, 1.1, seed)
    ar, ai, ir, ic = O.Port(g).assemble(O.PHYS_AC, freq, vp, rho)
    rc, ap, aidx, ax, az, _ = triplet_to_col(g.n, g.n, ir, ic, ar, ai)
    assert rc == 0
    ax[:ar.size] = ar
    az[:ai.size] = ai
    M = sp.csc_matrix((ax + 1j * az, aidx, ap), shape=(g.n, g.n))
    return g, ap, aidx, ax, az, M, (ar, ai, ir, ic)


# ------------------------------------------------------------- host (no GPU)
def test_triplet_to_col_matches_scipy_with_duplicates():
    rng = np.random.default_rng(5)
    n_row, n_col, nz = 37, 29, 400
    ti = rng.integers(0, n_row, nz)
    tj = rng.integers(0, n_col, nz)
    tx = rng.standard_normal(nz)
    tz = rng.standard_normal(nz)
    rc, ap, ai, ax, az, mp = triplet_to_col(n_row, n_col, ti, tj, tx, tz, want_map=True)
    assert rc == 0
    S = sp.coo_matrix((tx + 1j * tz, (ti, tj)), shape=(n_row, n_col)).tocsc()
    S.sum_duplicates()
    S.sort_indices()
    nnz = ap[-1]
    assert nnz == S.nnz
    np.testing.assert_array_equal(ap, S.indptr)
    np.testing.assert_array_equal(ai[:nnz], S.indices)
    np.testing.assert_allclose(ax[:nnz] + 1j * az[:nnz], S.data, rtol=0, atol=1e-12)
    # Map: every triplet lands on its (row, col) slot
    for k in range(nz):
        p = mp[k]
        assert ai[p] == ti[k] and ap[tj[k]] <= p < ap[tj[k] + 1]


def test_triplet_to_col_packed_and_pattern_only():
    rng = np.random.default_rng(6)
    n, nz = 20, 90
    ti, tj = rng.integers(0, n, nz), rng.integers(0, n, nz)
    v = rng.standard_normal(nz) + 1j * rng.standard_normal(nz)
    packed_in = np.stack([v.real, v.imag], axis=1).ravel()
    rc, ap, ai, ax, _, _ = triplet_to_col(n, n, ti, tj, packed_in, None, packed=True)
    assert rc == 0
    S = sp.coo_matrix((v, (ti, tj)), shape=(n, n)).tocsc()
    S.sum_duplicates()
    S.sort_indices()
    nnz = ap[-1]
    np.testing.assert_allclose(ax[:2 * nnz:2] + 1j * ax[1:2 * nnz:2], S.data, atol=1e-12)
    rc, ap2, ai2, _, _, _ = triplet_to_col(n, n, ti, tj)
    assert rc == 0
    np.testing.assert_array_equal(ap2, ap)
    np.testing.assert_array_equal(ai2[:nnz], ai[:nnz])


def test_triplet_to_col_errors():
    rc = triplet_to_col(4, 4, [0, 4], [0, 1], np.ones(2), np.zeros(2))[0]
    assert rc == _lib.UMFPACK_ERROR_invalid_matrix
    rc = triplet_to_col(0, 4, [0], [0], np.ones(1), np.zeros(1))[0]
    assert rc == -6
    assert b"positive" in umf().gm_umfpack_last_error()


def test_reference_pattern_is_csr_pattern():
    """The stencil pattern is symmetric: the CSC structure built from the
    reference's row-major triplets equals their CSR structure, which is why
    overwriting the values in triplet order hands UMFPACK M = A^T."""
    g, ap, aidx, ax, az, M, (ar, ai, ir, ic) = reference_flow_matrix(33, 27, 10.0, 5, 20.0, 0)
    A = OS.assembled_matrix(g, ar, ai, ir, ic)
    np.testing.assert_array_equal(ap, A.indptr)
    np.testing.assert_array_equal(aidx[:ap[-1]], A.indices)
    assert abs(M - OS.operator(A, 0)).max() == 0


def test_symbolic_detects_grid_and_rejects_others():
    g, ap, aidx, ax, az, M, _ = reference_flow_matrix(31, 23, 10.0, 4, 15.0, 1)
    sym = vp_t()
    info = np.zeros(90)
    rc = umf().umfpack_zi_symbolic(g.n, g.n, P(ap), P(aidx), P(ax), P(az), ctypes.byref(sym), None, P(info))
    assert rc == 0 and info[0] == 0 and sym.value
    umf().umfpack_zi_free_symbolic(ctypes.byref(sym))
    assert not sym.value
    # a tridiagonal matrix is no 9-point grid matrix
    T = sp.diags([np.ones(49), 2 * np.ones(50), np.ones(49)], [-1, 0, 1]).tocsc()
    T.sort_indices()
    tp, ti = T.indptr.astype(np.int32), T.indices.astype(np.int32)
    rc = umf().umfpack_zi_symbolic(50, 50, P(tp), P(ti), None, None, ctypes.byref(sym), None, P(info))
    assert rc == _lib.UMFPACK_ERROR_invalid_matrix and info[0] == rc
    # a grid matrix with one far-away entry
    B = (M + sp.csc_matrix(([1.0], ([g.n - 1], [0])), shape=M.shape)).tocsc()
    B.sort_indices()
    bp, bi = B.indptr.astype(np.int32), B.indices.astype(np.int32)
    rc = umf().umfpack_zi_symbolic(g.n, g.n, P(bp), P(bi), None, None, ctypes.byref(sym), None, None)
    assert rc == _lib.UMFPACK_ERROR_invalid_matrix
    assert b"outside the 9-point stencil" in umf().gm_umfpack_last_error()
    # rectangular
    rc = umf().umfpack_zi_symbolic(g.n, g.n - 1, P(ap), P(aidx), None, None, ctypes.byref(sym), None, None)
    assert rc == _lib.UMFPACK_ERROR_invalid_matrix


def test_numeric_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    g, ap, aidx, ax, az, M, _ = reference_flow_matrix(21, 19, 10.0, 3, 15.0, 2)
    sym, num = vp_t(), vp_t()
    assert umf().umfpack_zi_symbolic(g.n, g.n, P(ap), P(aidx), P(ax), P(az), ctypes.byref(sym), None, None) == 0
    rc = umf().umfpack_zi_numeric(P(ap), P(aidx), P(ax), P(az), sym, ctypes.byref(num), None, None)
    umf().umfpack_zi_free_symbolic(ctypes.byref(sym))
    assert rc < 0 and not num.value
    assert b"no CUDA device" in umf().gm_umfpack_last_error()


# ------------------------------------------------------------------- GPU
def _factor(g, ap, aidx, ax, az):
    sym, num = vp_t(), vp_t()
    assert umf().umfpack_zi_symbolic(g.n, g.n, P(ap), P(aidx), P(ax), P(az), ctypes.byref(sym), None, None) == 0
    rc = umf().umfpack_zi_numeric(P(ap), P(aidx), P(ax), P(az), sym, ctypes.byref(num), None, None)
    umf().umfpack_zi_free_symbolic(ctypes.byref(sym))
    assert rc == 0, umf().gm_umfpack_last_error()
    return num


def _solve(num, sys_, b, g, packed=False):
    info = np.zeros(90)
    if packed:
        bp = np.stack([b.real, b.imag], axis=1).ravel()
        xp = np.zeros(2 * g.n)
        rc = umf().umfpack_zi_solve(sys_, None, None, None, None, P(xp), None, P(bp), None, num, None, P(info))
        x = xp[0::2] + 1j * xp[1::2]
    else:
        br, bi = np.ascontiguousarray(b.real), np.ascontiguousarray(b.imag)
        xr, xi = np.zeros(g.n), np.zeros(g.n)
        rc = umf().umfpack_zi_solve(sys_, None, None, None, None, P(xr), P(xi), P(br), P(bi), num, None, P(info))
        x = xr + 1j * xi
    assert rc == 0 and info[0] == 0, umf().gm_umfpack_last_error()
    return x


@pytest.mark.gpu
@pytest.mark.parametrize("sys_", [0, 1, 2], ids=["A", "At_conj", "Aat"])
def test_reference_flow_solves_match_superlu(sys_):
    g, ap, aidx, ax, az, M, _ = reference_flow_matrix(61, 47, 10.0, 8, 18.0, 3)
    num = _factor(g, ap, aidx, ax, az)
    rng = np.random.default_rng(sys_)
    op = {0: M, 1: M.conj().T, 2: M.T}[sys_].tocsc()
    ref = OS.DirectSolver(op)
    for packed in (False, True):
        b = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
        x = _solve(num, sys_, b, g, packed=packed)
        xr = ref.solve(b)
        assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= 1e-10
        assert np.linalg.norm(op @ x - b) / np.linalg.norm(b) <= 1e-10
    umf().umfpack_zi_free_numeric(ctypes.byref(num))
    assert not num.value


@pytest.mark.gpu
def test_driver_sequence_over_frequencies_reuses_engines():
    """The drivers' per-frequency sequence (triplet_to_col, symbolic,
    numeric, free_symbolic, one solve per shot, free_numeric) twice, then
    two live numeric objects at once: each keeps its own factors."""
    nums = []
    for freq in (10.0, 22.0):
        g, ap, aidx, ax, az, M, _ = reference_flow_matrix(45, 39, 10.0, 6, freq, 4)
        num = _factor(g, ap, aidx, ax, az)
        ref = OS.DirectSolver(M)
        for s in range(3):
            b = np.zeros(g.n, complex)
            b[(s + 1) * g.n // 4] = 1.0 / 100.0
            x = _solve(num, 0, b, g)
            xr = ref.solve(b)
            assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= 1e-10
        nums.append((num, M, g))
    for num, M, g in nums:
        b = np.ones(g.n) + 0.5j
        x = _solve(num, 0, b, g)
        xr = OS.DirectSolver(M).solve(b)
        assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= 1e-10
        umf().umfpack_zi_free_numeric(ctypes.byref(num))


@pytest.mark.gpu
def test_numeric_rejects_a_different_pattern():
    g, ap, aidx, ax, az, M, _ = reference_flow_matrix(41, 33, 10.0, 5, 15.0, 5)
    sym, num = vp_t(), vp_t()
    assert umf().umfpack_zi_symbolic(g.n, g.n, P(ap), P(aidx), P(ax), P(az), ctypes.byref(sym), None, None) == 0
    ap2 = ap.copy()
    ap2[-1] -= 1
    rc = umf().umfpack_zi_numeric(P(ap2), P(aidx), P(ax), P(az), sym, ctypes.byref(num), None, None)
    assert rc == _lib.UMFPACK_ERROR_different_pattern and not num.value
    rc = umf().umfpack_zi_solve(7, None, None, None, None, None, None, None, None, None, None, None)
    assert rc == -3   # invalid Numeric object comes first
    umf().umfpack_zi_free_symbolic(ctypes.byref(sym))
