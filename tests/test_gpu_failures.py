"""Failure paths of the engine (the reference ignores every UMFPACK status,
src/AC/forward_shot_AC.c:41,58,61,88; the engine's status codes replace
them).  Every failure here is made on the host or by a wait that nothing
signals: no GPU fault, trap or hang is provoked."""
import ctypes

import numpy as np
import pytest

from germaine_b200 import GM_OP_EXACT, GM_PREC_C64_IR, GM_PREC_FP64, Engine, GmError, _lib
from tests.models import random_smooth

pytestmark = pytest.mark.gpu


def _model(nx, ny, seed=1):
    return random_smooth(nx, ny, 1500.0, 3500.0, seed), np.full((ny, nx), 1000.0, np.float32)


@pytest.mark.parametrize("bad", ["nan-vp", "zero-vp", "zero-rho"])
@pytest.mark.parametrize("precision", [GM_PREC_FP64, GM_PREC_C64_IR], ids=["fp64", "c64"])
def test_nonfinite_material_is_reported(bad, precision):
    """NaN material, or material whose operator coefficients overflow
    (1/(rho vp^2) or 1/rho infinite), stops the factorisation with
    GM_ERROR_NONFINITE."""
    nx, ny = 40, 30
    vp, rho = _model(nx, ny)
    if bad == "zero-rho":
        rho[12, 17] = 0.0               # b = 1/rho = inf
    elif bad == "zero-vp":
        vp[12, 17] = 0.0                # ivp2 = 1/(rho vp^2) = inf
    else:
        vp[12, 17] = np.nan
    with Engine(nx, ny, 10.0, 6, precision=precision, leaf_max=16) as e:
        e.set_model(vp, rho)
        with pytest.raises(GmError) as ex:
            e.factor([9.0])
        assert ex.value.code == _lib.GM_ERROR_NONFINITE
        # the engine stays usable: a clean model factorises afterwards
        vp2, rho2 = _model(nx, ny)
        e.set_model(vp2, rho2)
        assert e.factor([9.0]) == _lib.GM_OK


def test_zero_pivot_is_perturbed_and_counted():
    """A zeroed operator row (M[r][*] = 0 through gm_factor_values) makes a
    zero pivot: the static pivot is replaced, counted, and the factorisation
    returns GM_WARNING_PERTURBED; the singular system then cannot meet the
    residual target (GM_WARNING_NOT_CONVERGED), with finite results."""
    nx, ny = 36, 28
    vp, rho = _model(nx, ny, seed=3)
    with Engine(nx, ny, 10.0, 6, op_mode=GM_OP_EXACT, leaf_max=16, ir_max_iter=2) as e:
        e.set_model(vp, rho)
        e.factor([8.0])
        ar, ai, ir, ic = e.triplets(0)
    n = nx * ny
    re = np.zeros((9, n)); im = np.zeros((9, n))
    qof = {di + dj * nx: (di + 1) + 3 * (dj + 1) for dj in (-1, 0, 1) for di in (-1, 0, 1)}
    for a, b, r, c in zip(ar, ai, ir, ic):
        q = qof[int(c) - int(r)]
        re[q, r] = a
        im[q, r] = b
    row = 14 * nx + 17
    re[:, row] = 0.0
    im[:, row] = 0.0
    lib = _lib.load()
    with Engine(nx, ny, 10.0, 6, op_mode=GM_OP_EXACT, leaf_max=16, ir_max_iter=2) as e:
        rc = lib.gm_factor_values(e._h, 1, _lib.ptr(np.ascontiguousarray(re)), _lib.ptr(np.ascontiguousarray(im)))
        assert rc == _lib.GM_WARNING_PERTURBED
        e.nf = 1
        assert e.stats()["perturbed_pivots"] >= 1
        b = np.zeros((1, n, 2), complex)
        b[0, 100, 0] = 1.0
        b[0, row, 1] = 1.0j              # the zeroed row's equation 0 = 1j has no solution
        x = e.solve(b)
        assert e.last_status == _lib.GM_WARNING_NOT_CONVERGED
        assert np.all(np.isfinite(x))


def test_bounded_wait_runs_out():
    """The tcgen05 kernels' bounded mbarrier wait, on an mbarrier that no
    thread signals: it gives up after the given polls and reports the
    timeout instead of hanging (the factorisation turns such a report into
    GM_ERROR_CUDA)."""
    lib = _lib.load()
    out = ctypes.c_int(-1)
    for polls in (1, 1000, 100_000):
        _lib.check(lib.gm_wait_probe(0, polls, ctypes.byref(out)))
        assert out.value == 1
    assert lib.gm_wait_probe(0, 0, ctypes.byref(out)) == _lib.GM_ERROR_INVALID
