"""Pins the oracle: the C restatement (oracle/port.c) against the reference's
own sources compiled into oracle/_ref, and both against the committed golden
fixtures (tests/golden/, made by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import oracle as O
from tests.models import inclusion_ac, random_smooth, te_model

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def _materials(physics, g, seed):
    if physics == O.PHYS_AC:
        vp, rho = inclusion_ac(g.nx, g.ny, g.dh, g.npml)
        return vp * random_smooth(g.nx, g.ny, 0.9, 1.1, seed), rho
    if physics == O.PHYS_SH:
        return random_smooth(g.nx, g.ny, 800, 2500, seed), random_smooth(g.nx, g.ny, 1500, 2600, seed + 1)
    return te_model(g.nx, g.ny, seed)


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference tree absent)")


@needs_ref
@pytest.mark.parametrize("physics,freq", [(1, 15.0), (2, 7.0), (4, 2e8)])
@pytest.mark.parametrize("s,fs", [(0.0, 0), (1.3, 1)])
def test_port_assembly_equals_reference(physics, freq, s, fs):
    g = O.Grid(nx=45, ny=33, dh=10.0 if physics != 4 else 0.025, npml=8, free_surf=fs, s=s)
    m0, m1 = _materials(physics, g, 5)
    a = O.Port(g).assemble(physics, freq, m0, m1)
    b = O.Ref(g).assemble(physics, freq, m0, m1)
    for x, y in zip(a, b):
        assert np.array_equal(_bits(x), _bits(y))
    assert np.array_equal(_bits(O.Port(g).pml(freq)), _bits(O.Ref(g).pml(freq)))


@needs_ref
def test_port_nonzero_equals_reference():
    for nx, ny in [(241, 141), (3, 3), (10, 4)]:
        g = O.Grid(nx=nx, ny=ny, dh=10.0, npml=1)
        assert O.Ref(g).nonzero() == g.nonzero
    assert O.Grid(nx=241, ny=141, dh=10.0, npml=20).nonzero == 303541


@needs_ref
@pytest.mark.parametrize("physics", [1, 4])
def test_port_shot_arithmetic_equals_reference(physics):
    g = O.Grid(nx=40, ny=30, dh=10.0, npml=6, s=0.4)
    P, R = O.Port(g), O.Ref(g)
    f = 9.0 if physics == 1 else 1.5e8
    for xs, ys in [(55.0, 30.0), (104.9, 25.1), (0.0, 0.0)]:
        a, b = P.rhs_source(physics, f, xs, ys), R.rhs_source(physics, f, xs, ys)
        assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(_bits(a[1]), _bits(b[1]))
    rng = np.random.default_rng(2)
    x = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
    pa, pb = P.vec2mat(x), R.vec2mat(x)
    assert np.array_equal(pa[0], pb[0]) and np.array_equal(pa[1], pb[1])
    rx = np.arange(1, 25, dtype=np.int32); ry = np.full(rx.size, 2, np.int32)
    sa = np.zeros(rx.size, np.float32); sb = np.zeros(rx.size, np.float32)
    sa2 = np.zeros(rx.size, np.float32); sb2 = np.zeros(rx.size, np.float32)
    P.calc_seis(pa[0], pa[1], rx, ry, 1, 1, 1, sa, sa2)
    R.calc_seis(pb[0], pb[1], rx, ry, 1, 1, 1, sb, sb2, 1)
    assert np.array_equal(sa, sb) and np.array_equal(sa2, sb2)
    obs_r = rng.standard_normal(rx.size).astype(np.float32)
    obs_i = rng.standard_normal(rx.size).astype(np.float32)
    for stf_inv in (0, 1):
        for misfit in (1, 2, 3):
            la, ra, ia, wa = P.calc_res(sa, sa2, obs_r, obs_i, stf_inv, 1, misfit)
            lb, rb, ib, wb = R.calc_res(sb, sb2, obs_r, obs_i, stf_inv, 1, misfit)
            assert np.array_equal(ra, rb) and np.array_equal(ia, ib) and np.array_equal(wa, wb)
            if stf_inv == 1:
                assert la == lb
    ad, bd = P.rhs_adj(ra, ia, rx, ry), R.rhs_adj(rb, ib, rx, ry)
    assert np.array_equal(ad[0], bd[0]) and np.array_equal(ad[1], bd[1])
    stf = np.array([0.7, -0.3], np.float32)
    vp = random_smooth(g.nx, g.ny, 1500, 3000, 1); rho = random_smooth(g.nx, g.ny, 1000, 2000, 2)
    fr, fi, lr, li = (rng.standard_normal(g.n).astype(np.float32) for _ in range(4))
    if physics == 1:
        ga = np.zeros(g.n, np.float32); gb = np.zeros(g.n, np.float32)
        P.ass_grad_ac(f, stf, fr, fi, lr, li, vp, rho, ga)
        R.ass_grad_ac(f, stf, fr, fi, lr, li, vp, rho, gb)
        assert np.array_equal(ga, gb)
        P.cp_grad_frame(ga); R.cp_grad_frame(gb)
        assert np.array_equal(ga, gb)
    else:
        ga = np.zeros(g.n, np.float32); gb = np.zeros(g.n, np.float32)
        ea = np.zeros(g.n, np.float32); eb = np.zeros(g.n, np.float32)
        P.ass_grad_te(f, stf, fr, fi, lr, li, ga, ea)
        R.ass_grad_te(f, stf, fr, fi, lr, li, gb, eb)
        assert np.array_equal(ga, gb) and np.array_equal(ea, eb)


def _golden_files():
    """assembly / solve fixtures (the post-processing and file-format fixtures have their own tests)"""
    return (sorted(f for f in os.listdir(GOLDEN)
                   if f.endswith(".npz") and not f.startswith(("postproc_", "files_")))
            if os.path.isdir(GOLDEN) else [])


@pytest.mark.parametrize("fname", _golden_files())
def test_port_against_golden(fname):
    """Fixtures generated from the reference's own compiled sources."""
    d = np.load(os.path.join(GOLDEN, fname))
    g = O.Grid(nx=int(d["nx"]), ny=int(d["ny"]), dh=float(d["dh"]), npml=int(d["npml"]),
               free_surf=int(d["free_surf"]), a0_pml=float(d["a0_pml"]), s=float(d["s"]))
    physics, freq = int(d["physics"]), float(d["freq"])
    a = O.Port(g).assemble(physics, freq, d["m0"], d["m1"])
    assert np.array_equal(_bits(a[0]), _bits(d["Ar"])) and np.array_equal(_bits(a[1]), _bits(d["Ai"]))
    assert np.array_equal(a[2], d["irow"]) and np.array_equal(a[3], d["icol"])
    assert np.array_equal(_bits(O.Port(g).pml(freq)), _bits(d["pml"]))
    if "x" in d:
        from oracle import sparse as OS
        M = OS.operator(OS.assembled_matrix(g, *a))
        x = OS.DirectSolver(M).solve(d["b"])
        assert np.linalg.norm(x - d["x"]) / np.linalg.norm(d["x"]) < 1e-12


def gauss_cases():
    d = np.load(os.path.join(GOLDEN, "postproc_gauss_filt.npz"))
    out = []
    for k in range(int(d["ncases"])):
        nx, ny, dh, vref, fc, fs0, fs1 = d[f"case_{k}"]
        out.append((int(nx), int(ny), float(dh), float(vref), float(fc), float(fs0), float(fs1), d[f"grad_{k}"],
                    d[f"out_{k}"]))
    return out


def test_port_gauss_filt_against_golden():
    """gauss_filt (src/gauss_filt.c:10-141): the restatement is bit-identical
    to the reference's output stored in the fixture, including the filter-off
    and unnormalised (negative size) cases."""
    for nx, ny, dh, vref, fc, fs0, fs1, grad, ref in gauss_cases():
        g = O.Grid(nx=nx, ny=ny, dh=dh, npml=6)
        assert np.array_equal(_bits(O.Port(g).gauss_filt(grad, vref, fc, fs0, fs1)), _bits(ref))


@needs_ref
@pytest.mark.parametrize("fs0,fs1", [(0.5, 0.5), (0.25, 0.6), (1.1, 0.15), (-0.3, 0.3), (0.4, -0.2)])
def test_port_gauss_filt_equals_reference(fs0, fs1):
    g = O.Grid(nx=57, ny=43, dh=12.5, npml=6)
    grad = np.random.default_rng(3).standard_normal((43, 57)).astype(np.float32)
    a = O.Port(g).gauss_filt(grad, 2500.0, 4.0, fs0, fs1)
    b = O.Ref(g).gauss_filt(grad, 2500.0, 4.0, fs0, fs1)
    assert np.array_equal(_bits(a), _bits(b))


def hess_cases():
    d = np.load(os.path.join(GOLDEN, "postproc_apply_hess.npz"))
    out = []
    for k in range(int(d["ncases"])):
        nx, ny, eps = d[f"case_{k}"]
        out.append((int(nx), int(ny), float(np.float32(eps)), d[f"grad_{k}"], d[f"hess_{k}"], d[f"out_{k}"],
                    float(d[f"max_{k}"])))
    return out


def test_port_apply_hess_against_golden():
    """apply_hess_AC (src/AC/apply_hess_AC.c:11-40): the restatement is
    bit-identical to the reference's output stored in the fixture (negative
    and zero Hessian entries, EPS_HESS = 0 included)."""
    for nx, ny, eps, grad, hess, ref, mx in hess_cases():
        g = O.Grid(nx=nx, ny=ny, dh=10.0, npml=4)
        out, m = O.Port(g).apply_hess(grad, hess, eps)
        assert np.array_equal(_bits(out), _bits(ref)) and m == mx


@needs_ref
@pytest.mark.parametrize("eps", [0.005, 0.3, 1e-7])
def test_port_apply_hess_equals_reference(eps):
    g = O.Grid(nx=41, ny=35, dh=10.0, npml=4)
    rng = np.random.default_rng(9)
    grad = rng.standard_normal((35, 41)).astype(np.float32)
    hess = (rng.standard_normal((35, 41)) * 1e-4).astype(np.float32)
    a, ma = O.Port(g).apply_hess(grad, hess, eps)
    b, mb = O.Ref(g).apply_hess(grad, hess, eps)
    assert np.array_equal(_bits(a), _bits(b)) and ma == mb


# ---- l-BFGS (src/LBFGS.c, src/TE/LBFGS_TE.c) ----
from tests import lbfgs_cases as LC  # noqa: E402


@needs_ref
def test_port_lbfgs_ac_equals_reference(short_tmp):
    """Six iterations with NLBFGS = 3 (two rotations): every direction bit-identical."""
    g, m = LC.grid(), 3
    seq = LC.sequence(g, 1, 6, seed=1)
    port, ref = O.PortLbfgs(g, m, 1), O.RefLbfgs(g, m, 1, os.path.join(short_tmp, "j"))
    a = LC.run(lambda f, p, it, gr, gm, md, h: port.step(f, p, gr, gm, md), port.rotate, m, seq)
    b = LC.run(lambda f, p, it, gr, gm, md, h: ref.step_ac(it, p, gr, gm, md), ref.rotate, m, seq)
    for x, y in zip(a, b):
        assert np.array_equal(_bits(x), _bits(y))
    assert np.array_equal(_bits(port.y), _bits(ref.y)) and np.array_equal(_bits(port.s), _bits(ref.s))


@needs_ref
@pytest.mark.parametrize("with_hess", [False, True], ids=["gamma", "hessian"])
def test_port_lbfgs_te_equals_reference(short_tmp, with_hess):
    g, m, norms, eps = LC.grid(free_surf=1), 2, (0.01, 8.85e-11), 0.005
    seq = LC.sequence(g, 2, 5, seed=2)
    port, ref = O.PortLbfgs(g, m, 2), O.RefLbfgs(g, m, 2, os.path.join(short_tmp, "j"))
    hs = (lambda h: h) if with_hess else (lambda h: None)
    a = LC.run(lambda f, p, it, gr, gm, md, h: port.step(f, p, gr, gm, LC.normalise(md, norms), hs(h), eps),
               port.rotate, m, seq)
    b = LC.run(lambda f, p, it, gr, gm, md, h: ref.step_te(f, p, gr, gm, md, norms, hs(h), eps), ref.rotate, m, seq)
    for x, y in zip(a, b):
        assert np.array_equal(_bits(x), _bits(y))


@needs_ref
def test_port_check_descent_sums_equal_reference():
    g = LC.grid()
    rng = np.random.default_rng(8)
    hg = rng.standard_normal((g.ny, g.nx)).astype(np.float32)
    gr = rng.standard_normal((g.ny, g.nx)).astype(np.float32)
    R = O.Ref(g)
    nom, den = R.lib.ref_dotp_matrix(hg.ravel(), gr.ravel()), R.lib.ref_dotp_matrix(gr.ravel(), gr.ravel())
    p = O.PortLbfgs(g, 1, 1).check_descent(hg, gr)
    assert _bits(np.float32(p)) == _bits(np.float32(-np.float32(nom)) / np.float32(den))


# ---- precond (src/precond.c) ----
def precond_cases():
    d = np.load(os.path.join(GOLDEN, "postproc_precond.npz"))
    out = []
    for k in range(int(d["ncases"])):
        nx, ny, npml, fs, spat, hor, gt2, tfile = (int(v) for v in d[f"case_{k}"])
        g = O.Grid(nx=nx, ny=ny, dh=10.0, npml=npml, free_surf=fs)
        out.append((g, dict(spatfilter=spat, vref=2000.0, fc_low=5.0, fsg=0.3, fsg1=0.5, taper_hor=hor, gradt2=gt2,
                            taper=d[f"taper_{k}"] if tfile else None), d[f"grad_{k}"], d[f"out_{k}"]))
    return out


def test_port_precond_against_golden():
    """precond (src/precond.c:10-24): gauss_filt, taper_grad_hor and
    taper_grad_file, incl. its overwrite of the top interior rows with a
    free surface; bit-identical to the reference's output in the fixture."""
    for g, kw, grad, ref in precond_cases():
        assert np.array_equal(_bits(O.Port(g).precond(grad, **kw)), _bits(ref))


@needs_ref
def test_port_precond_equals_reference(short_tmp):
    rng = np.random.default_rng(21)
    for fs in (0, 1):
        g = O.Grid(nx=40, ny=28, dh=12.5, npml=5, free_surf=fs)
        nx0, ny0 = g.nx - 2 * g.npml, g.ny - g.npml - g.fsshift
        grad = rng.standard_normal((g.ny, g.nx)).astype(np.float32)
        taper = rng.uniform(0, 1, nx0 * ny0).astype(np.float32)
        kw = dict(spatfilter=1, vref=2500.0, fc_low=4.0, fsg=0.2, fsg1=0.6, taper_hor=1, gradt2=3, taper=taper)
        a = O.Port(g).precond(grad, **kw)
        b = O.Ref(g).precond(short_tmp, grad, **kw)
        assert np.array_equal(_bits(a), _bits(b))


# ---- per-shot gradient tapers (src/taper_grad_shot.c, src/taper_grad_shot1.c) ----
def shot_taper_cases():
    d = np.load(os.path.join(GOLDEN, "postproc_shot_taper.npz"))
    out = []
    for k in range(int(d["ncases"])):
        nx, ny, dh, radius, fs = d[f"case_{k}"]
        out.append((int(nx), int(ny), float(np.float32(dh)), float(np.float32(radius)), int(fs), d[f"grad_{k}"],
                    d[f"sx_{k}"], d[f"sy_{k}"], d[f"rx_{k}"], d[f"ry_{k}"], d[f"rad_{k}"], d[f"sq_{k}"]))
    return out


def test_shot_tapers_against_golden():
    """taper_grad_shot for every shot and taper_grad_shot1: the restatement
    (oracle/port.c) and the product's host drop-ins (gm_taper_grad_shot,
    gm_taper_grad_shot1) are bit-identical to the reference's outputs stored
    in the fixture."""
    from germaine_b200 import taper_grad_shot, taper_grad_shot1
    for nx, ny, dh, radius, fs, grad, sx, sy, rx, ry, rad, sq in shot_taper_cases():
        g = O.Grid(nx=nx, ny=ny, dh=dh, npml=4)
        port = O.Port(g)
        for s in range(len(sx)):
            assert np.array_equal(_bits(port.taper_grad_shot(grad, radius, sx, sy, rx, ry, s)), _bits(rad[s]))
            got = taper_grad_shot(grad.reshape(ny, nx), dh, radius, sx, sy, rx, ry, s)
            assert np.array_equal(_bits(got.ravel()), _bits(rad[s]))
        assert np.array_equal(_bits(port.taper_grad_shot1(grad, fs, sx, sy, rx, ry)), _bits(sq))
        got = taper_grad_shot1(grad.reshape(ny, nx), dh, fs, sx, sy, rx, ry)
        assert np.array_equal(_bits(got.ravel()), _bits(sq))
        assert np.any(rad != grad[None, :]) and np.any(sq != grad)


@needs_ref
@pytest.mark.parametrize("radius", [25.0, 62.5, 150.0])
def test_shot_tapers_equal_reference(radius):
    """Random interior geometries, sources off the grid nodes, overlapping
    receiver tapers: restatement, product and reference bit-identical."""
    from germaine_b200 import taper_grad_shot, taper_grad_shot1
    g = O.Grid(nx=57, ny=43, dh=12.5, npml=6)
    rng = np.random.default_rng(int(radius))
    grad = rng.standard_normal(g.n).astype(np.float32)
    sx = (rng.uniform(4, 53, 3) * g.dh).astype(np.float32)
    sy = (rng.uniform(4, 39, 3) * g.dh).astype(np.float32)
    rx = rng.integers(4, 53, 11).astype(np.int32)
    ry = rng.integers(4, 39, 11).astype(np.int32)
    ref, port = O.Ref(g), O.Port(g)
    for s in range(3):
        want = ref.taper_grad_shot(grad, radius, sx, sy, rx, ry, s)
        assert np.array_equal(_bits(port.taper_grad_shot(grad, radius, sx, sy, rx, ry, s)), _bits(want))
        got = taper_grad_shot(grad.reshape(g.ny, g.nx), g.dh, radius, sx, sy, rx, ry, s)
        assert np.array_equal(_bits(got.ravel()), _bits(want))
    for fs in (0, 1, 2):
        want = ref.taper_grad_shot1(grad, fs, sx, sy, rx, ry)
        assert np.array_equal(_bits(port.taper_grad_shot1(grad, fs, sx, sy, rx, ry)), _bits(want))
        got = taper_grad_shot1(grad.reshape(g.ny, g.nx), g.dh, fs, sx, sy, rx, ry)
        assert np.array_equal(_bits(got.ravel()), _bits(want))


def test_shot_taper_squares_clipped_at_the_edge():
    """Squares that cross the grid edge (where the reference writes past its
    arrays) are clipped: restatement and product agree, nothing outside the
    grid is touched."""
    from germaine_b200 import GmError, taper_grad_shot1
    g = O.Grid(nx=20, ny=16, dh=5.0, npml=3)
    grad = np.arange(g.n, dtype=np.float32) + 1
    sx = np.array([0.0, 97.0], np.float32)
    sy = np.array([2.0, 78.0], np.float32)
    rx = np.array([1, 20], np.int32)
    ry = np.array([16, 1], np.int32)
    a = O.Port(g).taper_grad_shot1(grad, 2, sx, sy, rx, ry)
    b = taper_grad_shot1(grad.reshape(g.ny, g.nx), g.dh, 2, sx, sy, rx, ry).ravel()
    assert np.array_equal(_bits(a), _bits(b))
    assert np.count_nonzero(b == np.float32(1e-5)) > 0
    with pytest.raises(GmError):
        taper_grad_shot1(grad.reshape(g.ny, g.nx), g.dh, -1, sx, sy, rx, ry)
    from germaine_b200 import taper_grad_shot
    with pytest.raises(GmError):      # shot index out of range
        taper_grad_shot(grad.reshape(g.ny, g.nx), g.dh, 10.0, sx, sy, rx, ry, 2)
    with pytest.raises(GmError):      # radius must be positive
        taper_grad_shot(grad.reshape(g.ny, g.nx), g.dh, 0.0, sx, sy, rx, ry, 0)


# ---- Tikhonov regularisation of TE FWI (src/TE/Tikhonov_cost_TE.c, Tikhonov_grad_TE.c) ----
def tikhonov_cases():
    d = np.load(os.path.join(GOLDEN, "postproc_tikhonov_te.npz"))
    out = []
    for k in range(int(d["ncases"])):
        c = d[f"case_{k}"]
        nx, ny, idx, idy = int(c[0]), int(c[1]), int(c[3]), int(c[4])
        dh, n1, n2, b1, b2, l1, l2, misfit = (float(np.float32(v)) for v in (c[2], *c[5:12]))
        out.append((nx, ny, dh, idx, idy, n1, n2, b1, b2, l1, l2, misfit, d[f"sig_{k}"], d[f"eps_{k}"],
                    d[f"gsig_{k}"], d[f"geps_{k}"], float(d[f"cost_{k}"]), d[f"gs_{k}"], d[f"ge_{k}"]))
    return out


def test_tikhonov_te_against_golden():
    """gm_tikhonov_cost_te / gm_tikhonov_grad_te bit-identical to the
    reference's outputs stored in the fixture (IDX/IDY subsampling, one
    LAMBDA zero, both zero)."""
    from germaine_b200 import tikhonov_cost_te, tikhonov_grad_te
    for (nx, ny, dh, idx, idy, n1, n2, b1, b2, l1, l2, misfit, sig, eps, gsig, geps, cost, gs,
         ge) in tikhonov_cases():
        got = tikhonov_cost_te(sig, eps, misfit, dh, n1, n2, b1, b2, l1, l2, idx, idy)
        assert np.float32(got).view(np.uint32) == np.float32(cost).view(np.uint32)
        a, b = tikhonov_grad_te(gsig, geps, sig, eps, dh, n1, n2, b1, b2, l1, l2, idx, idy)
        assert np.array_equal(_bits(a.ravel()), _bits(gs)) and np.array_equal(_bits(b.ravel()), _bits(ge))


@needs_ref
@pytest.mark.parametrize("idx,idy,lam", [(1, 1, (0.2, 0.9)), (3, 2, (0.0, 5e-4)), (1, 4, (2.0, 0.0))])
def test_tikhonov_te_equals_reference(idx, idy, lam):
    from germaine_b200 import GmError, tikhonov_cost_te, tikhonov_grad_te
    g = O.Grid(nx=45, ny=31, dh=0.04, npml=5)
    rng = np.random.default_rng(idx * 10 + idy)
    sig = rng.uniform(1e-4, 2e-2, (g.ny, g.nx)).astype(np.float32)
    eps = (rng.uniform(2, 30, (g.ny, g.nx)) * 8.8541878e-12).astype(np.float32)
    gsig = rng.standard_normal((g.ny, g.nx)).astype(np.float32)
    geps = rng.standard_normal((g.ny, g.nx)).astype(np.float32)
    args = (0.01, 8.85e-11, 1.0, 0.5, *lam)
    ref = O.Ref(g)
    want = ref.tikhonov_cost_te(sig, eps, 12.5, *args, idx, idy)
    got = tikhonov_cost_te(sig, eps, 12.5, g.dh, *args, idx, idy)
    assert np.float32(got).view(np.uint32) == np.float32(want).view(np.uint32)
    ws, we = ref.tikhonov_grad_te(gsig, geps, sig, eps, *args, idx, idy)
    gs, ge = tikhonov_grad_te(gsig, geps, sig, eps, g.dh, *args, idx, idy)
    assert np.array_equal(_bits(gs.ravel()), _bits(ws)) and np.array_equal(_bits(ge.ravel()), _bits(we))
    with pytest.raises(GmError):
        tikhonov_cost_te(sig, eps, 12.5, g.dh, 0.0, 8.85e-11, 1.0, 0.5, *lam)     # MAT1_NORM = 0
