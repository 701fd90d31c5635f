"""Gradient post-processing on the device (gm_gauss_filt, the SPATFILTER = 1
smoothing of precond(), src/gauss_filt.c:10-141): bit-identical to the
reference's output in the committed fixture and to the C restatement, for
host and device buffers and in place."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from germaine_b200 import _lib, gauss_filt
from tests.test_oracle_pin import GOLDEN, _bits, gauss_cases

pytestmark = pytest.mark.gpu


def test_gauss_filt_matches_reference_fixture():
    for nx, ny, dh, vref, fc, fs0, fs1, grad, ref in gauss_cases():
        out = gauss_filt(grad, dh, vref, fc, fs0, fs1)
        assert np.array_equal(_bits(out), _bits(ref)), (nx, ny, fs0, fs1)


@pytest.mark.parametrize("fs0,fs1", [(0.5, 0.5), (0.15, 0.9), (-0.3, 0.3)])
def test_gauss_filt_device_buffers_and_in_place(fs0, fs1):
    import torch
    nx, ny, dh, vref, fc = 200, 90, 25.0, 3000.0, 3.0
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=10)
    grad = np.random.default_rng(5).standard_normal((ny, nx)).astype(np.float32)
    want = O.Port(g).gauss_filt(grad, vref, fc, fs0, fs1)
    d = torch.from_numpy(grad).cuda()
    lib = _lib.load()
    _lib.check(lib.gm_gauss_filt(0, nx, ny, dh, vref, fc, fs0, fs1, _lib.ptr(d), _lib.ptr(d)))   # in place
    assert np.array_equal(_bits(d.cpu().numpy()), _bits(want))


def test_gauss_filt_rejects_bad_arguments():
    lib = _lib.load()
    g = np.zeros((4, 4), np.float32)
    assert lib.gm_gauss_filt(0, 0, 4, 10.0, 2000.0, 5.0, 0.5, 0.5, _lib.ptr(g), _lib.ptr(g)) == _lib.GM_ERROR_INVALID
    assert lib.gm_gauss_filt(0, 4, 4, 10.0, 2000.0, 0.0, 0.5, 0.5, _lib.ptr(g), _lib.ptr(g)) == _lib.GM_ERROR_INVALID


def test_precond_matches_reference_fixture():
    """gm_precond (precond: gauss_filt, taper_grad_hor, taper_grad_file)
    bit-identical to the reference's output in the committed fixture."""
    from germaine_b200 import precond
    from tests.test_oracle_pin import precond_cases
    for g, kw, grad, ref in precond_cases():
        out = precond(grad, g.npml, g.free_surf, g.dh, spatfilter=kw["spatfilter"], vref=kw["vref"],
                      fc_low=kw["fc_low"], filt_size_grad=kw["fsg"], filt_size_grad1=kw["fsg1"],
                      taper_hor=kw["taper_hor"], gradt2=kw["gradt2"], taper=kw["taper"])
        assert np.array_equal(_bits(out), _bits(ref)), (g.nx, g.ny, g.free_surf, kw["spatfilter"])
