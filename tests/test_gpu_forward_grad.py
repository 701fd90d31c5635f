"""Forward modelling (seismograms, wavefields) and the FWI objective/gradient
on the GPU vs the FP64 oracle (SuperLU on M = A^T + FP64 restatements of
vec2mat / calc_seis / calc_res / RHS_source_AC_adj / ass_grad / cp_grad_frame).

Tolerances: solution-level quantities in FP64 (the returned FP64 gradient)
1e-8 relative; complex64 / float outputs 2e-6 relative (their rounding)."""
import numpy as np
import pytest

import oracle as O
from oracle import sparse as OS
from germaine_b200 import (GM_PHYS_AC, GM_PHYS_SH, GM_PHYS_TE, GM_PREC_C64_IR, GM_PREC_FP64, GM_SYS_A, GM_SYS_AT,
                           Engine, GmError)
from tests.models import inclusion_ac, random_smooth, te_model

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _case(physics, seed=0):
    if physics == GM_PHYS_TE:
        nx, ny, dh, npml, freqs = 46, 38, 0.05, 8, [1.0e8, 2.2e8]
        m0, m1 = te_model(nx, ny, seed)
    elif physics == GM_PHYS_SH:
        nx, ny, dh, npml, freqs = 50, 36, 10.0, 8, [6.0, 13.0]
        m0, m1 = random_smooth(nx, ny, 900, 2400, seed), random_smooth(nx, ny, 1600, 2500, seed + 1)
    else:
        nx, ny, dh, npml, freqs = 64, 44, 10.0, 10, [7.0, 15.0]
        vp, rho = inclusion_ac(nx, ny, dh, npml, radius=60.0)
        m0, m1 = vp * random_smooth(nx, ny, 0.9, 1.1, seed), rho
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    nx0 = nx - 2 * npml
    xs = np.linspace(2 * dh, (nx0 - 3) * dh, 5).astype(np.float32)
    ys = np.full(5, 3 * dh, np.float32)
    rx = np.arange(1, nx0 - 1, dtype=np.int32)
    ry = np.full(rx.size, 3, np.int32)
    return g, m0, m1, freqs, xs, ys, rx, ry


def oracle_forward(g, physics, m0, m1, freqs, xs, ys, trans_adj=False):
    port = O.Port(g)
    sols, solvers = [], []
    for f in freqs:
        A = OS.assembled_matrix(g, *port.assemble(physics, f, m0, m1))
        ds = OS.DirectSolver(OS.operator(A))
        solvers.append(ds)
        sols.append(ds.solve(OS.spike_rhs(g, physics, f, xs, ys, port)))
    return np.stack(sols), solvers


@pytest.mark.parametrize("physics", [GM_PHYS_AC, GM_PHYS_SH, GM_PHYS_TE], ids=["ac", "sh", "te"])
@pytest.mark.parametrize("precision", [GM_PREC_FP64, GM_PREC_C64_IR], ids=["fp64", "c64ir"])
def test_forward_seismograms_and_fields(physics, precision):
    g, m0, m1, freqs, xs, ys, rx, ry = _case(physics)
    with Engine(g.nx, g.ny, g.dh, g.npml, physics=physics, precision=precision, leaf_max=32) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        seis, field = e.forward(xs, ys, rx, ry, want_field=True)
    X, _ = oracle_forward(g, physics, m0, m1, freqs, xs, ys)
    idx = [OS.receiver_read_index(g, int(a), int(b)) for a, b in zip(rx, ry)]
    for i in range(len(freqs)):
        fld = OS.vec2mat(X[i].T)                       # [ns][n] complex128
        assert _rel(field[i], fld) < 2e-6
        assert _rel(seis[i], fld[:, idx]) < 2e-6
        assert np.all(field[i][:, -1] == 0)            # x[N] is defined as 0


def test_forward_field_layout_matches_reference_vec2mat():
    """The wavefield output is byte-for-byte the reference's vec2mat of the
    engine's own FP64 solution (float cast + one-slot shift)."""
    g, m0, m1, freqs, xs, ys, rx, ry = _case(GM_PHYS_AC)
    with Engine(g.nx, g.ny, g.dh, g.npml) as e:
        e.set_model(m0, m1)
        e.factor(freqs[:1])
        _, field = e.forward(xs, ys, rx, ry, want_field=True)
        B = OS.spike_rhs(g, 1, freqs[0], xs, ys)
        x = e.solve(B)                                  # [n][ns]
    conv = O.Ref(g) if O.ref_available() else O.Port(g)
    for s in range(len(xs)):
        pr, pi = conv.vec2mat(x[:, s])
        assert np.array_equal(field[0][s].real, pr) and np.array_equal(field[0][s].imag, pi)


def oracle_grad(g, physics, m0, m1, freqs, xs, ys, rx, ry, obs, stf_inv, misfit, taper=None, invmat=1):
    X, solvers = oracle_forward(g, physics, m0, m1, freqs, xs, ys)
    idx = [OS.receiver_read_index(g, int(a), int(b)) for a, b in zip(rx, ry)]
    kadj = [OS.adjoint_index(g, int(a), int(b)) for a, b in zip(rx, ry)]
    dh2 = float(np.float32(g.dh) * np.float32(g.dh))
    l2 = 0.0
    Xa = np.zeros_like(X)
    stfu = np.zeros((len(freqs), len(xs)), complex)
    for i in range(len(freqs)):
        fld = OS.vec2mat(X[i].T)
        Badj = np.zeros((g.n, len(xs)), complex)
        for s in range(len(xs)):
            li, res, w = OS.residual_fp64(fld[s, idx], obs[i, s], stf_inv, misfit, invmat)
            l2 += li
            stfu[i, s] = w / abs(w)
            for t, k in enumerate(kadj):
                Badj[k, s] = np.conj(res[t]) / dh2
        Xa[i] = solvers[i].solve(Badj, trans=(physics == GM_PHYS_TE))
    g0, g1 = OS.gradient_fp64(g, physics, freqs, X, Xa, stfu, vp=m0, rho=m1, taper=taper)
    return g0, g1, 0.5 * l2


def _observed(g, physics, m0, m1, freqs, xs, ys, rx, ry, seed=5):
    """Observed data from a perturbed model, with a few exact zeros to
    exercise the reference's adjoint-source zeroing."""
    p0 = m0 * random_smooth(g.nx, g.ny, 0.95, 1.05, seed)
    X, _ = oracle_forward(g, physics, p0, m1, freqs, xs, ys)
    idx = [OS.receiver_read_index(g, int(a), int(b)) for a, b in zip(rx, ry)]
    obs = np.stack([OS.vec2mat(X[i].T)[:, idx] for i in range(len(freqs))]).astype(np.complex64)
    obs[:, :, 3] = 0
    obs[:, 1, 7] = -1e-3 - 2e-3j     # both parts negative: zeroed adjoint source (calc_res_AC.c:82-85)
    return obs


@pytest.mark.parametrize("physics,stf_inv,misfit", [(GM_PHYS_AC, 0, 1), (GM_PHYS_AC, 1, 1), (GM_PHYS_AC, 0, 2),
                                                     (GM_PHYS_AC, 0, 3), (GM_PHYS_TE, 0, 1), (GM_PHYS_TE, 1, 1)],
                         ids=["ac-l2", "ac-stf", "ac-log", "ac-phase", "te-l2", "te-stf"])
def test_gradient_matches_fp64_oracle(physics, stf_inv, misfit):
    g, m0, m1, freqs, xs, ys, rx, ry = _case(physics, seed=1)
    obs = _observed(g, physics, m0, m1, freqs, xs, ys, rx, ry)
    if misfit == 2:
        obs[:, :, 3] = 1e-3 + 1e-3j      # log misfit needs non-zero data
    with Engine(g.nx, g.ny, g.dh, g.npml, physics=physics, leaf_max=32) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        g0f, g1f, l2, _ = e.grad_obj(xs, ys, rx, ry, obs, stf_inv=stf_inv, misfit=misfit)
        g0, g1 = e.gradient_fp64()
        l2o = e.obj(xs, ys, rx, ry, obs, stf_inv=stf_inv, misfit=misfit)
    r0, r1, rl2 = oracle_grad(g, physics, m0, m1, freqs, xs, ys, rx, ry, obs, stf_inv, misfit)
    assert _rel(g0, r0) < 1e-8
    assert _rel(g0f, r0) < 2e-6
    if physics == GM_PHYS_TE:
        assert _rel(g1, r1) < 1e-8
        assert _rel(g1f, r1) < 2e-6
    assert abs(l2 - rl2) / rl2 < 2e-6 and abs(l2o - rl2) / rl2 < 2e-6


@pytest.mark.parametrize("physics", [GM_PHYS_AC, GM_PHYS_TE], ids=["ac", "te"])
@pytest.mark.parametrize("mode", [1, 2], ids=["radial", "squares"])
def test_gradient_shot_taper(physics, mode):
    """SWS_TAPER_CIRCULAR_PER_SHOT = 1 (taper_grad_shot) and 2
    (taper_grad_shot1) applied per shot inside the gradient stack, against
    the FP64 oracle with the same per-shot coefficients; the tapered points
    are checked on their own (the squares' 1e-5 is small against the
    gradient), the others are the untapered gradient."""
    g, m0, m1, freqs, xs, ys, rx, ry = _case(physics, seed=3)
    obs = _observed(g, physics, m0, m1, freqs, xs, ys, rx, ry)
    radius, filtsize = float(np.float32(3.5 * g.dh)), 1
    with Engine(g.nx, g.ny, g.dh, g.npml, physics=physics, leaf_max=32) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        e.set_shot_taper(mode, radius, filtsize)
        e.grad_obj(xs, ys, rx, ry, obs)
        t0, t1 = e.gradient_fp64()
        e.set_shot_taper(0)
        e.grad_obj(xs, ys, rx, ry, obs)
        u0, u1 = e.gradient_fp64()
        with pytest.raises(GmError):
            e.set_shot_taper(3)
        with pytest.raises(GmError):
            e.set_shot_taper(1, 0.0)
    taper = OS.shot_taper(g, mode, xs, ys, rx, ry, radius, filtsize)
    r0, r1, _ = oracle_grad(g, physics, m0, m1, freqs, xs, ys, rx, ry, obs, 0, 1, taper=taper)
    touched = np.any(taper[1] != 1.0, axis=0) if mode == 1 else taper[1]
    assert 0 < touched.sum() < g.n
    pairs = [(t0, u0, r0)] + ([(t1, u1, r1)] if physics == GM_PHYS_TE else [])
    for t, u, r in pairs:
        assert _rel(t, r) < 1e-8
        assert _rel(t[touched], r[touched]) < 1e-8
        assert _rel(t[~touched], u[~touched]) < 1e-12
        assert _rel(u[touched], t[touched]) > 1e-3       # the taper changed those points


def test_gradient_mixed_precision_within_1e6():
    g, m0, m1, freqs, xs, ys, rx, ry = _case(GM_PHYS_AC, seed=2)
    obs = _observed(g, GM_PHYS_AC, m0, m1, freqs, xs, ys, rx, ry)
    with Engine(g.nx, g.ny, g.dh, g.npml, precision=GM_PREC_C64_IR, leaf_max=32) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        e.grad_obj(xs, ys, rx, ry, obs)
        g0, _ = e.gradient_fp64()
    r0, _, _ = oracle_grad(g, GM_PHYS_AC, m0, m1, freqs, xs, ys, rx, ry, obs, 0, 1)
    assert _rel(g0, r0) < 1e-6


def test_adjoint_dot_product():
    """<M^-T s, r> = <s, M^-1 r> (non-conjugate bilinear form) through the
    engine's two solve orientations."""
    g, m0, m1, freqs, *_ = _case(GM_PHYS_TE)
    rng = np.random.default_rng(3)
    s = rng.standard_normal((1, g.n, 1)) + 1j * rng.standard_normal((1, g.n, 1))
    r = rng.standard_normal((1, g.n, 1)) + 1j * rng.standard_normal((1, g.n, 1))
    with Engine(g.nx, g.ny, g.dh, g.npml, physics=GM_PHYS_TE) as e:
        e.set_model(m0, m1)
        e.factor(freqs[:1])
        a = e.solve(s, sys=GM_SYS_AT)
        b = e.solve(r, sys=GM_SYS_A)
    lhs = np.sum(a * r)
    rhs = np.sum(s * b)
    assert abs(lhs - rhs) / abs(rhs) < 1e-11


def test_duplicate_receivers_last_wins_and_bad_geometry():
    g, m0, m1, freqs, xs, ys, rx, ry = _case(GM_PHYS_AC, seed=4)
    rx = np.concatenate([rx, rx[:3]]).astype(np.int32)     # three receivers twice
    ry = np.concatenate([ry, ry[:3]]).astype(np.int32)
    obs = _observed(g, GM_PHYS_AC, m0, m1, freqs, xs, ys, rx, ry)
    with Engine(g.nx, g.ny, g.dh, g.npml) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        e.grad_obj(xs, ys, rx, ry, obs)
        g0, _ = e.gradient_fp64()
        with pytest.raises(GmError):
            e.forward(np.array([1e9], np.float32), np.array([0.0], np.float32), rx, ry)
        with pytest.raises(GmError):
            e.forward(xs, ys, np.array([10_000], np.int32), np.array([1], np.int32))
    r0, _, _ = oracle_grad(g, GM_PHYS_AC, m0, m1, freqs, xs, ys, rx, ry, obs, 0, 1)
    assert _rel(g0, r0) < 1e-8


def test_state_errors():
    g, m0, m1, freqs, xs, ys, rx, ry = _case(GM_PHYS_AC)
    with Engine(g.nx, g.ny, g.dh, g.npml) as e:
        with pytest.raises(GmError):
            e.factor(freqs)                          # no model yet
        e.set_model(m0, m1)
        with pytest.raises(GmError):
            e.forward(xs, ys, rx, ry)                # no factorisation yet
        with pytest.raises(GmError):
            e.factor([-1.0])


@pytest.mark.parametrize("physics,stf_inv", [(GM_PHYS_AC, 0), (GM_PHYS_AC, 1), (GM_PHYS_TE, 0)],
                         ids=["ac", "ac-stf", "te"])
def test_rtm_image_invmat2(physics, stf_inv):
    """INVMAT = 2 (RTM_FD_AC's use of grad_obj_AC): the residual is the
    observed data (src/AC/calc_res_AC.c:77), back-propagated and stacked
    like a gradient; misfit = 0.5 sum |obs|^2 of the non-zeroed samples."""
    g, m0, m1, freqs, xs, ys, rx, ry = _case(physics, seed=6)
    obs = _observed(g, physics, m0, m1, freqs, xs, ys, rx, ry)
    with Engine(g.nx, g.ny, g.dh, g.npml, physics=physics, leaf_max=32) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        e.set_invmat(2)
        _, _, l2, _ = e.grad_obj(xs, ys, rx, ry, obs, stf_inv=stf_inv)
        g0, g1 = e.gradient_fp64()
        l2o = e.obj(xs, ys, rx, ry, obs, stf_inv=stf_inv)
        e.set_invmat(1)
        e.grad_obj(xs, ys, rx, ry, obs, stf_inv=stf_inv)
        f0, _ = e.gradient_fp64()
        with pytest.raises(GmError):
            e.set_invmat(3)
    r0, r1, rl2 = oracle_grad(g, physics, m0, m1, freqs, xs, ys, rx, ry, obs, stf_inv, 1, invmat=2)
    assert _rel(g0, r0) < 1e-8
    if physics == GM_PHYS_TE:
        assert _rel(g1, r1) < 1e-8
    assert abs(l2 - rl2) / rl2 < 2e-6 and abs(l2o - rl2) / rl2 < 2e-6
    assert _rel(f0, g0) > 1e-3          # the FWI gradient differs


@pytest.mark.parametrize("physics", [GM_PHYS_AC, GM_PHYS_TE], ids=["ac", "te"])
def test_source_wavelet_amplitudes(physics):
    """READ_WAVELET = 1: each frequency's spike carries the wavelet's DFT
    amplitude over DH^2 (src/AC/RHS_source_AC.c:40-55), for the forward
    fields and the gradient."""
    g, m0, m1, freqs, xs, ys, rx, ry = _case(physics, seed=7)
    amp = np.array([0.8 - 0.3j, -0.25 + 1.1j], np.complex64)[:len(freqs)]
    with Engine(g.nx, g.ny, g.dh, g.npml, physics=physics, leaf_max=32) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        e.set_source_wavelet(amp)
        seis, _ = e.forward(xs, ys, rx, ry)
        X = e.wavefield_fp64(0, len(xs))
        e.set_source_wavelet(amp[:1])                # wrong count for the batch
        with pytest.raises(GmError):
            e.forward(xs, ys, rx, ry)
        e.set_source_wavelet(None)
        seis1, _ = e.forward(xs, ys, rx, ry)
    port = O.Port(g)
    dh2 = np.float32(g.dh) * np.float32(g.dh)
    idx = [OS.receiver_read_index(g, int(a), int(b)) for a, b in zip(rx, ry)]
    for i, f in enumerate(freqs):
        A = OS.assembled_matrix(g, *port.assemble(physics, f, m0, m1))
        ds = OS.DirectSolver(OS.operator(A))
        B = np.zeros((g.n, len(xs)), complex)
        for s in range(len(xs)):
            k = OS.source_index(g, float(xs[s]), float(ys[s]))
            B[k, s] = complex(np.float32(amp[i].real) / dh2, np.float32(amp[i].imag) / dh2)
        Xr = ds.solve(B)
        assert _rel(X[i], Xr) < 1e-10
        assert _rel(seis[i], OS.vec2mat(Xr.T)[:, idx]) < 2e-6
    assert _rel(seis1, seis) > 1e-2
