"""Threshold pivoting inside 32-row pivot blocks, restated in numpy over the
engine's own symbolic analysis (test infrastructure: the arithmetic of the
GPU kernels in plain form) and checked against SuperLU on both solves.

The factorisation exchanges rows only inside a front's current 32-pivot
block and only in the block's own columns and those to its right; the
multipliers of earlier blocks stay in equation order ("lazy" form).  The
forward pass of M x = b therefore takes a block's right-hand-side rows in
pivot order when it reaches the block (after the earlier blocks' updates),
and the backward pass of M^T x = b writes a block's result back in equation
order before the earlier blocks use it.  tau = 1 exchanges whenever a larger
entry exists, so every block of every front above the smallest is
exercised."""
import numpy as np
import pytest

import oracle as O
from oracle import sparse as OS
from tests.test_symbolic import stencil_values, symbolic

NB = 32


def factor(S, A9, tau):
    F, P = [None] * S["nn"], [None] * S["nn"]
    swaps = 0
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
        perm = np.arange(s)   # perm[k]: the front row (equation order) at pivot position k
        for k in range(s):
            k0 = (k // NB) * NB
            kend = min(s, k0 + NB)
            j = k + int(np.argmax(np.abs(Fv[k:kend, k])))
            if j != k and abs(Fv[k, k]) < tau * abs(Fv[j, k]):
                Fv[[k, j], k0:] = Fv[[j, k], k0:]   # the block's columns and those right of it only
                perm[[k, j]] = perm[[j, k]]
                swaps += 1
            Fv[k + 1:, k] /= Fv[k, k]
            Fv[k + 1:, k + 1:] -= np.outer(Fv[k + 1:, k], Fv[k, k + 1:])
        F[v], P[v] = Fv, perm
    return F, P, swaps


def solve(S, F, P, b):
    """M x = b: forward pass with the block gathers, then U x = y."""
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
        for k0 in range(0, s, NB):
            k1 = min(s, k0 + NB)
            w[k0:k1] = w[k0 + P[v][k0:k1] - k0]   # the block's rows in pivot order
            for k in range(k0, k1):
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


def solve_t(S, F, P, b):
    """M^T x = b: U^T z = b forward, then L^T backward with the block scatters."""
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
        U = F[v]
        for k in range(s):   # U^T: column k of U is row k of U^T
            w[k] /= U[k, k]
            w[k + 1:] -= U[k, k + 1:] * w[k]
        x[vs[:s]] = w[:s]
        W[v] = w[s:]
    for v in reversed(range(S["nn"])):
        s = S["npiv"][v]
        vs = S["vars"][S["var_off"][v]:S["var_off"][v + 1]]
        L = F[v]
        t = x[vs[:s]] - L[s:, :s].T @ x[vs[s:]]
        for k0 in reversed(range(0, s, NB)):
            k1 = min(s, k0 + NB)
            for k in reversed(range(k0, k1)):   # L_bb^T, unit diagonal
                t[k0:k] -= L[k, k0:k] * t[k]
            blk = t[k0:k1].copy()
            t[k0 + P[v][k0:k1] - k0] = blk   # back to equation order
            t[:k0] -= L[k0:k1, :k0].T @ t[k0:k1]   # earlier blocks read it in equation order
        x[vs[:s]] = t
    return x


@pytest.mark.parametrize("shape", [(41, 33, 16), (66, 38, 12), (35, 71, 20)])
def test_block_pivoting_replay_matches_superlu(shape):
    nx, ny, leaf = shape
    g = O.Grid(nx=nx, ny=ny, dh=10.0, npml=2)
    rng = np.random.default_rng(nx * ny)
    vp = rng.uniform(1500, 3000, g.n).astype(np.float32)
    rho = rng.uniform(1000, 2000, g.n).astype(np.float32)
    trip = O.Port(g).assemble(1, 9.0, vp, rho)
    A9 = stencil_values(g, *trip)
    S = symbolic(nx, ny, leaf)
    assert S["npiv"].max() > NB   # at least one front with more than one pivot block
    F, P, swaps = factor(S, A9, tau=1.0)
    assert swaps > 0
    M = OS.operator(OS.assembled_matrix(g, *trip))
    ds = OS.DirectSolver(M)
    b = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
    x = solve(S, F, P, b)
    xr = ds.solve(b)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-10
    xt = solve_t(S, F, P, b)
    xtr = ds.solve(b, trans=True)
    assert np.linalg.norm(xt - xtr) / np.linalg.norm(xtr) < 1e-10
