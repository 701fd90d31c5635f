"""tcgen05 complex-FP32 GEMM (3xTF32 split products, TMEM accumulator) vs
the CUDA-core kernel and a complex128 reference, over ragged shapes."""
import ctypes

import numpy as np
import pytest

from germaine_b200 import _lib

pytestmark = pytest.mark.gpu

SHAPES = [  # m, n, k, lda_pad
    (128, 64, 16, 0), (1, 1, 1, 0), (130, 70, 33, 5), (300, 129, 97, 0), (64, 200, 227, 3),
    (454, 454, 210, 0), (7, 300, 5, 1), (256, 64, 0, 0),
]


def _run(backend, shapes, seed):
    import torch
    rng = np.random.default_rng(seed)
    hostA, hostB, hostC, dev = [], [], [], []
    dims = []
    for (m, n, k, pad) in shapes:
        lda, ldb, ldc = m + pad, k + pad, m + pad
        A = (rng.standard_normal((lda, max(k, 1))) + 1j * rng.standard_normal((lda, max(k, 1)))).astype(np.complex64)
        B = (rng.standard_normal((max(ldb, 1), n)) + 1j * rng.standard_normal((max(ldb, 1), n))).astype(np.complex64)
        C = (rng.standard_normal((ldc, n)) + 1j * rng.standard_normal((ldc, n))).astype(np.complex64)
        hostA.append(A); hostB.append(B); hostC.append(C)
        # column-major device copies
        dA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").view(np.float32).copy()).cuda()
        dB = torch.from_numpy(np.asfortranarray(B).ravel(order="F").view(np.float32).copy()).cuda()
        dC = torch.from_numpy(np.asfortranarray(C).ravel(order="F").view(np.float32).copy()).cuda()
        dev.append((dA, dB, dC))
        dims += [m, n, k, lda, max(ldb, 1), ldc]
    P = ctypes.c_void_p * len(shapes)
    pa = P(*[d[0].data_ptr() for d in dev]); pb = P(*[d[1].data_ptr() for d in dev]); pc = P(*[d[2].data_ptr() for d in dev])
    dims = np.array(dims, np.int32)
    lib = _lib.load()
    _lib.check(lib.gm_cgemm_sub_c64(0, backend, len(shapes), dims.ctypes.data, pa, pb, pc))
    out = []
    for (m, n, k, pad), (dA, dB, dC), A, B, C in zip(shapes, dev, hostA, hostB, hostC):
        got = dC.cpu().numpy().view(np.complex64).reshape(C.shape[1], C.shape[0]).T
        ref = C.astype(np.complex128).copy()
        ref[:m, :] -= A[:m, :k].astype(np.complex128) @ B[:k, :].astype(np.complex128)
        out.append((got, ref, A, B, m, n, k))
    return out


@pytest.mark.parametrize("backend", [0, 1], ids=["cuda-cores", "tcgen05"])
def test_cgemm_matches_reference(backend):
    for got, ref, A, B, m, n, k in _run(backend, SHAPES, seed=backend):
        scale = np.abs(A[:m, :k]).max(initial=0) * np.abs(B[:k, :]).max(initial=0) * max(k, 1) + 1.0
        err = np.abs(got - ref).max() / scale
        assert err < 2e-6, f"{m}x{n}x{k}: error {err:.2e}"
        # rows beyond m (the lda padding) are untouched
        assert np.array_equal(got[m:], ref[m:].astype(np.complex64))


def test_tcgen05_agrees_with_cuda_cores():
    a = _run(0, SHAPES[:5], seed=7)
    b = _run(1, SHAPES[:5], seed=7)
    for (g0, ref, *_), (g1, *_ ) in zip(a, b):
        assert np.abs(g0 - g1).max() / (np.abs(ref).max() + 1) < 1e-5
