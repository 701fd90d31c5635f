"""gm_solve_noalloc: the block solve + refinement for callers that cannot
allocate device memory while solving (cudaFree stalls every stream of the
device; a caller with a fixed, pre-reserved memory budget has nothing left to
allocate from).  Its workspaces live in one fixed-size device array inside the
library instead of cudaMalloc'd buffers.  Checked through the C-ABI against
gm_solve on the same factors, on two calls in a row (the second one runs over
the first one's leftovers in the shared array), with free device memory
unchanged across the first call after the engine was created and factorised;
host pointers and overlapping b / x are refused before any kernel runs."""
import ctypes

import numpy as np
import pytest

from germaine_b200 import GM_PREC_C64_IR, GM_PREC_FP64, GM_SYS_A, GM_SYS_AT, Engine, _lib
from tests.models import inclusion_ac, random_smooth

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _case():
    nx, ny, dh, npml = 47, 35, 10.0, 8
    vp, rho = inclusion_ac(nx, ny, dh, npml, radius=50.0)
    vp = vp * random_smooth(nx, ny, 0.9, 1.1, 4)
    return nx, ny, dh, npml, vp, rho


@pytest.mark.parametrize("nrhs", [6, 40], ids=["one-slice", "two-slices"])
@pytest.mark.parametrize("precision", [GM_PREC_FP64, GM_PREC_C64_IR], ids=["fp64", "c64ir"])
@pytest.mark.parametrize("sys_", [GM_SYS_A, GM_SYS_AT], ids=["A", "At"])
def test_noalloc_solve_matches_gm_solve_twice(precision, sys_, nrhs):
    import torch
    nx, ny, dh, npml, vp, rho = _case()
    rng = np.random.default_rng(9)
    b = rng.standard_normal((2, nx * ny, nrhs)) + 1j * rng.standard_normal((2, nx * ny, nrhs))
    lib = _lib.load()
    b_d = torch.from_numpy(b.view(np.float64).copy()).cuda()
    x_d = torch.full_like(b_d, float("nan"))
    with Engine(nx, ny, dh, npml, precision=precision, leaf_max=24) as e:
        e.set_model(vp, rho)
        e.factor([8.0, 14.0])
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        rc = lib.gm_solve_noalloc(e._h, sys_, nrhs, _lib.ptr(b_d), _lib.ptr(x_d))
        _lib.check(rc)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, f"the first gm_solve_noalloc call took {free0 - free1} bytes of device memory"
        x_first = x_d.cpu().numpy().view(np.complex128).reshape(b.shape)
        x_ref = e.solve(b, sys=sys_)                      # gm_solve
        res_ref = e.stats()["ir_residual"]
        assert res_ref <= 1e-10
        assert _rel(x_first, x_ref) <= 1e-10
        for _ in range(2):
            x_d.fill_(float("nan"))
            torch.cuda.synchronize()
            rc = lib.gm_solve_noalloc(e._h, sys_, nrhs, _lib.ptr(b_d), _lib.ptr(x_d))
            _lib.check(rc)
            torch.cuda.synchronize()
            x = x_d.cpu().numpy().view(np.complex128).reshape(b.shape)
            assert _rel(x, x_ref) <= 1e-10
            assert e.stats()["ir_residual"] <= 1e-10


def test_noalloc_rejects_problems_beyond_the_scratch():
    import torch
    nx, ny, dh, npml = 120, 90, 10.0, 10
    vp = random_smooth(nx, ny, 1800, 2600, 1)
    rho = np.full((ny, nx), 1000.0, np.float32)
    lib = _lib.load()
    with Engine(nx, ny, dh, npml) as e:
        e.set_model(vp, rho)
        e.factor([6.0, 9.0, 12.0])
        nrhs = 64
        b_d = torch.zeros((3, nx * ny, 2 * nrhs), dtype=torch.float64, device="cuda")
        x_d = torch.zeros_like(b_d)
        rc = lib.gm_solve_noalloc(e._h, GM_SYS_A, nrhs, _lib.ptr(b_d), _lib.ptr(x_d))
        assert rc == _lib.GM_ERROR_INVALID
        assert b"scratch" in lib.gm_last_error()


def test_noalloc_rejects_host_and_overlapping_buffers():
    """Argument checks only: every call here returns before any kernel runs."""
    import torch
    nx, ny, dh, npml, vp, rho = _case()
    nrhs = 4
    lib = _lib.load()
    with Engine(nx, ny, dh, npml, leaf_max=24) as e:
        e.set_model(vp, rho)
        e.factor([8.0])
        cnt = nx * ny * nrhs * 2
        b_h = np.zeros(cnt, np.float64)
        x_h = np.zeros(cnt, np.float64)
        b_d = torch.zeros(cnt, dtype=torch.float64, device="cuda")
        x_d = torch.zeros(cnt, dtype=torch.float64, device="cuda")
        host_b = b_h.ctypes.data_as(ctypes.c_void_p)
        host_x = x_h.ctypes.data_as(ctypes.c_void_p)
        for b_ptr, x_ptr in ((host_b, _lib.ptr(x_d)), (_lib.ptr(b_d), host_x)):
            rc = lib.gm_solve_noalloc(e._h, GM_SYS_A, nrhs, b_ptr, x_ptr)
            assert rc == _lib.GM_ERROR_INVALID
            assert b"device" in lib.gm_last_error()
        both = torch.zeros(cnt + 8, dtype=torch.float64, device="cuda")
        for off in (0, 8):   # same buffer; x starting 4 complex values into b
            x_ptr = ctypes.c_void_p(both.data_ptr() + off * 8)
            rc = lib.gm_solve_noalloc(e._h, GM_SYS_A, nrhs, _lib.ptr(both), x_ptr)
            assert rc == _lib.GM_ERROR_INVALID
            assert b"overlap" in lib.gm_last_error()
