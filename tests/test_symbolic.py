"""Host symbolic analysis (nested dissection + extend-add maps), checked on
the CPU by replaying the multifrontal LU in numpy with the exported maps and
comparing the solution with SuperLU on the same operator."""
import ctypes

import numpy as np
import pytest

import oracle as O
from oracle import sparse as OS
from germaine_b200 import _lib


def symbolic(nx, ny, leaf):
    lib = _lib.load()
    h = ctypes.c_void_p()
    _lib.check(lib.gm_symbolic_create(nx, ny, leaf, ctypes.byref(h)))
    sz = np.zeros(16, np.int64)
    lib.gm_symbolic_sizes(h, sz.ctypes.data)
    n, nn, nl, nv, ft, ninv, nent, rt = (int(v) for v in sz[:8])

    def ex(w, cnt, dt):
        a = np.zeros(cnt, dt)
        _lib.check(lib.gm_symbolic_export(h, w, a.ctypes.data))
        return a

    S = dict(n=n, nn=nn, nl=nl, perm=ex(0, n, np.int32), iperm=ex(1, n, np.int32), npiv=ex(2, nn, np.int32),
             nfront=ex(3, nn, np.int32), parent=ex(4, nn, np.int32), height=ex(5, nn, np.int32),
             c0=ex(6, nn, np.int32), c1=ex(7, nn, np.int32), var_off=ex(8, nn + 1, np.int64),
             vars=ex(9, nv, np.int32), inv_off=ex(11, nn, np.int64), inv=ex(12, ninv, np.int32),
             ent_off=ex(13, nn + 1, np.int64), ent_pos=ex(14, nent, np.int32), ent_id=ex(15, nent, np.int32),
             front_total=ft, factor_flops=lib.gm_symbolic_flops(h, 0))
    lib.gm_symbolic_destroy(h)
    return S


def emulate_factor(S, A9):
    F = [None] * S["nn"]
    for v in range(S["nn"]):
        f, s = S["nfront"][v], S["npiv"][v]
        Fv = np.zeros((f, f), complex)
        for t, c in enumerate((S["c0"][v], S["c1"][v])):
            if c < 0:
                continue
            inv = S["inv"][S["inv_off"][v] + t * f:S["inv_off"][v] + (t + 1) * f]
            sc = S["npiv"][c]
            idx = np.nonzero(inv >= 0)[0]
            Fv[np.ix_(idx, idx)] += F[c][sc:, sc:][np.ix_(inv[idx], inv[idx])]
        e0, e1 = S["ent_off"][v], S["ent_off"][v + 1]
        Fv.T.flat[S["ent_pos"][e0:e1]] += A9.flat[S["ent_id"][e0:e1]]
        for k in range(s):
            Fv[k + 1:, k] /= Fv[k, k]
            Fv[k + 1:, k + 1:] -= np.outer(Fv[k + 1:, k], Fv[k, k + 1:])
        F[v] = Fv
    return F


def emulate_solve(S, F, b):
    x = b.astype(complex).copy()
    W = [None] * S["nn"]
    for v in range(S["nn"]):
        f, s = S["nfront"][v], S["npiv"][v]
        vs = S["vars"][S["var_off"][v]:S["var_off"][v + 1]]
        w = np.zeros(f, complex)
        w[:s] = x[vs[:s]]
        for t, c in enumerate((S["c0"][v], S["c1"][v])):
            if c < 0:
                continue
            inv = S["inv"][S["inv_off"][v] + t * f:S["inv_off"][v] + (t + 1) * f]
            idx = np.nonzero(inv >= 0)[0]
            w[idx] += W[c][inv[idx]]
        for k in range(s):
            w[k + 1:] -= F[v][k + 1:, k] * w[k]
        x[vs[:s]] = w[:s]
        W[v] = w[s:]
    for v in reversed(range(S["nn"])):
        s = S["npiv"][v]
        vs = S["vars"][S["var_off"][v]:S["var_off"][v + 1]]
        U = F[v]
        t = x[vs[:s]] - U[:s, s:] @ x[vs[s:]]
        for k in reversed(range(s)):
            t[k] /= U[k, k]
            t[:k] -= U[:k, k] * t[k]
        x[vs[:s]] = t
    return x


def stencil_values(g, ar, ai, ir, ic):
    A9 = np.zeros((9, g.n), complex)
    for q in range(9):
        di, dj = q % 3 - 1, q // 3 - 1
        sel = (ic - ir) == di + dj * g.nx
        # the column offset alone is ambiguous across row wraps; also match the grid step
        rx, cx = ir % g.nx, ic % g.nx
        sel &= (cx - rx) == di
        A9[q, ir[sel]] = ar[sel] + 1j * ai[sel]
    return A9


@pytest.mark.parametrize("shape", [(37, 29, 16), (5, 5, 4), (9, 4, 4), (60, 7, 12), (11, 40, 20), (3, 3, 4)])
def test_multifrontal_replay_matches_superlu(shape):
    nx, ny, leaf = shape
    g = O.Grid(nx=nx, ny=ny, dh=10.0, npml=1)
    rng = np.random.default_rng(nx * 100 + ny)
    vp = rng.uniform(1500, 3000, g.n).astype(np.float32)
    rho = rng.uniform(1000, 2000, g.n).astype(np.float32)
    trip = O.Port(g).assemble(1, 12.0, vp, rho)
    A9 = stencil_values(g, *trip)
    S = symbolic(nx, ny, leaf)
    assert sorted(S["perm"].tolist()) == list(range(g.n))
    assert np.array_equal(S["iperm"][S["perm"]], np.arange(g.n))
    F = emulate_factor(S, A9)
    b = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
    x = emulate_solve(S, F, b)
    M = OS.operator(OS.assembled_matrix(g, *trip))
    xr = OS.DirectSolver(M).solve(b)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-11


def test_structure_invariants():
    S = symbolic(120, 47, 32)
    nn = S["nn"]
    # postorder: children before parents, heights consistent
    for v in range(nn):
        for c in (S["c0"][v], S["c1"][v]):
            if c >= 0:
                assert c < v and S["parent"][c] == v and S["height"][c] < S["height"][v]
    # every matrix entry of the 9-point pattern is assigned exactly once
    nz = 9 * 120 * 47 - 6 * 120 - 6 * 47 + 4
    assert len(S["ent_id"]) == nz
    assert len(np.unique(S["ent_id"])) == nz
    assert S["factor_flops"] > 0


def test_bad_arguments():
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.gm_symbolic_create(0, 5, 16, ctypes.byref(h)) == _lib.GM_ERROR_INVALID
    assert b"bad argument" in lib.gm_last_error()
