"""Generates tests/golden/*.npz from the reference's OWN sources (compiled
into oracle/_ref by `make -C oracle ref`, where the reference tree is
present).  Each fixture holds one small seeded model, the reference's PML
profiles and assembled triplets (init_A_*_9p_pml) and, for the acoustic
cases, a right-hand side with its FP64 sparse solution on the operator
UMFPACK factorises (M = A^T; solved with SciPy SuperLU because UMFPACK is
not part of the reference tree); postproc_gauss_filt.npz holds gauss_filt
cases, postproc_apply_hess.npz apply_hess_AC cases, postproc_shot_taper.npz
taper_grad_shot / taper_grad_shot1 cases, postproc_tikhonov_te.npz
Tikhonov_cost_TE / Tikhonov_grad_TE cases and files_formats.npz the bytes
of the reference's seismogram and model files.
Run:  python tests/golden/make_golden.py [assembly] [gauss] [hess] [precond] [shot] [tikh] [files]
(no argument: all).
"""
import tempfile
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from oracle import sparse as OS  # noqa: E402
from tests.models import inclusion_ac, random_smooth, te_model  # noqa: E402

CASES = [
    # name, physics, nx, ny, dh, npml, free_surf, s, freq
    ("ac_inclusion_15hz", 1, 41, 31, 10.0, 10, 0, 0.0, 15.0),
    ("ac_freesurf_damped", 1, 36, 24, 25.0, 6, 1, 1.5, 6.0),
    ("sh_layers_7hz", 2, 34, 26, 10.0, 8, 0, 0.0, 7.0),
    ("te_gpr_200mhz", 4, 32, 30, 0.025, 8, 0, 0.0, 2.0e8),
]


def main():
    out = os.path.dirname(os.path.abspath(__file__))
    which = set(sys.argv[1:]) or {"assembly", "gauss", "hess", "precond", "shot", "tikh", "files"}
    if "assembly" in which:
        assembly_fixtures(out)
    if "gauss" in which:
        gauss_filt_fixture(out)
    if "hess" in which:
        apply_hess_fixture(out)
    if "precond" in which:
        precond_fixture(out)
    if "shot" in which:
        shot_taper_fixture(out)
    if "tikh" in which:
        tikhonov_fixture(out)
    if "files" in which:
        files_fixture(out)


def assembly_fixtures(out):
    for name, physics, nx, ny, dh, npml, fs, s, freq in CASES:
        g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml, free_surf=fs, s=s)
        if physics == 1:
            vp, rho = inclusion_ac(nx, ny, dh, npml, radius=3 * dh)
            m0, m1 = vp * random_smooth(nx, ny, 0.95, 1.05, 1), rho
        elif physics == 2:
            m0, m1 = random_smooth(nx, ny, 900, 2200, 2), random_smooth(nx, ny, 1600, 2500, 3)
        else:
            m0, m1 = te_model(nx, ny, 4)
        ref = O.Ref(g)
        ar, ai, ir, ic = ref.assemble(physics, freq, m0, m1)
        d = dict(nx=nx, ny=ny, dh=dh, npml=npml, free_surf=fs, a0_pml=g.a0_pml, s=s, physics=physics,
                 freq=freq, m0=m0, m1=m1, Ar=ar, Ai=ai, irow=ir, icol=ic, pml=ref.pml(freq))
        if physics == 1:
            rng = np.random.default_rng(7)
            b = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
            M = OS.operator(OS.assembled_matrix(g, ar, ai, ir, ic))
            d["b"] = b
            d["x"] = OS.DirectSolver(M).solve(b)
        np.savez_compressed(os.path.join(out, name + ".npz"), **d)
        print("wrote", name)


# gauss_filt (src/gauss_filt.c) cases: grid, VREF, FC_low, FILT_SIZE_GRAD, FILT_SIZE_GRAD1
GAUSS_CASES = [
    (61, 41, 10.0, 2000.0, 5.0, 0.5, 0.5),
    (61, 41, 10.0, 2000.0, 5.0, 0.3, 0.7),
    (45, 33, 25.0, 3000.0, 2.0, 0.2, 0.35),
    (61, 41, 10.0, 2000.0, 5.0, -0.4, 0.4),   # negative size: weights left unnormalised
    (61, 41, 10.0, 2000.0, 5.0, 0.0, 0.5),    # size 0: filter off
]


def gauss_filt_fixture(out):
    """postproc_gauss_filt.npz: seeded gradients and the reference's
    gauss_filt of each (case k in arrays with suffix _k)."""
    d = {"ncases": len(GAUSS_CASES)}
    rng = np.random.default_rng(11)
    for k, (nx, ny, dh, vref, fc, fs0, fs1) in enumerate(GAUSS_CASES):
        g = O.Grid(nx=nx, ny=ny, dh=dh, npml=6)
        grad = (rng.standard_normal((ny, nx)) * 1e-3).astype(np.float32)
        d[f"case_{k}"] = np.array([nx, ny, dh, vref, fc, fs0, fs1])
        d[f"grad_{k}"] = grad
        d[f"out_{k}"] = O.Ref(g).gauss_filt(grad, vref, fc, fs0, fs1)
    np.savez_compressed(os.path.join(out, "postproc_gauss_filt.npz"), **d)
    print("wrote postproc_gauss_filt")


# apply_hess_AC cases: grid, EPS_HESS
HESS_CASES = [(37, 29, 0.005), (50, 20, 0.1), (16, 16, 0.0)]


def apply_hess_fixture(out):
    """postproc_apply_hess.npz: seeded gradients and Hessians (positive, with
    zeros and negative entries) and the reference's apply_hess_AC of each:
    grad_k, hess_k, out_k, max_k (MAX_HESS), case_k = (nx, ny, eps)."""
    rng = np.random.default_rng(17)
    d = {"ncases": len(HESS_CASES)}
    for k, (nx, ny, eps) in enumerate(HESS_CASES):
        g = O.Grid(nx=nx, ny=ny, dh=10.0, npml=4)
        grad = rng.standard_normal((ny, nx)).astype(np.float32)
        hess = (np.exp(rng.uniform(-8, 3, (ny, nx))) * 1e-7).astype(np.float32)
        hess[rng.random((ny, nx)) < 0.05] = 0
        hess[rng.random((ny, nx)) < 0.03] *= -1
        if eps == 0.0:
            hess[hess == 0] = 1e-12     # EPS_HESS = 0 divides by hess itself
        o, mx = O.Ref(g).apply_hess(grad, hess, eps)
        d.update({f"case_{k}": np.array([nx, ny, eps]), f"grad_{k}": grad, f"hess_{k}": hess, f"out_{k}": o,
                  f"max_{k}": np.float32(mx)})
    np.savez_compressed(os.path.join(out, "postproc_apply_hess.npz"), **d)
    print("wrote postproc_apply_hess")


# per-shot taper cases: grid nx, ny, dh, SRTRADIUS, FILTSIZE, shots, receivers
SHOT_TAPER_CASES = [(61, 47, 12.5, 40.0, 1, 4, 9), (48, 40, 0.05, 0.18, 2, 3, 6), (35, 30, 10.0, 80.0, 0, 2, 5)]


def shot_taper_fixture(out):
    """postproc_shot_taper.npz: seeded one-shot gradients, interior source
    coordinates (metres, off the grid nodes) and receiver indices kept
    FILTSIZE + 1 points inside the grid, and the reference's taper_grad_shot
    of every shot (rad_k [ns][NY*NX]) and taper_grad_shot1 (sq_k);
    case_k = (nx, ny, dh, SRTRADIUS, FILTSIZE)."""
    rng = np.random.default_rng(23)
    d = {"ncases": len(SHOT_TAPER_CASES)}
    for k, (nx, ny, dh, radius, fs, ns, ntr) in enumerate(SHOT_TAPER_CASES):
        g = O.Grid(nx=nx, ny=ny, dh=dh, npml=4)
        grad = rng.standard_normal(ny * nx).astype(np.float32)
        lo = fs + 2
        sx = (rng.uniform(lo, nx - lo, ns) * dh).astype(np.float32)
        sy = (rng.uniform(lo, ny - lo, ns) * dh).astype(np.float32)
        rx = rng.integers(lo, nx - lo, ntr).astype(np.int32)
        ry = rng.integers(lo, ny - lo, ntr).astype(np.int32)
        ref = O.Ref(g)
        rad = np.stack([ref.taper_grad_shot(grad, radius, sx, sy, rx, ry, s) for s in range(ns)])
        sq = ref.taper_grad_shot1(grad, fs, sx, sy, rx, ry)
        d.update({f"case_{k}": np.array([nx, ny, dh, radius, fs]), f"grad_{k}": grad, f"sx_{k}": sx, f"sy_{k}": sy,
                  f"rx_{k}": rx, f"ry_{k}": ry, f"rad_{k}": rad, f"sq_{k}": sq})
    np.savez_compressed(os.path.join(out, "postproc_shot_taper.npz"), **d)
    print("wrote postproc_shot_taper")


# Tikhonov cases: grid nx, ny, dh, IDX, IDY, MAT1_NORM, MAT2_NORM, BETA_MAT1, BETA_MAT2, LAMBDA_1, LAMBDA_2
TIKH_CASES = [(37, 29, 0.05, 1, 1, 0.01, 8.85e-11, 1.0, 1.0, 0.3, 0.7),
              (40, 33, 0.025, 2, 3, 0.005, 1.77e-10, 0.5, 2.0, 1e-3, 0.0),
              (21, 18, 0.1, 1, 1, 0.01, 8.85e-11, 1.0, 1.0, 0.0, 0.0)]


def tikhonov_fixture(out):
    """postproc_tikhonov_te.npz: seeded TE models (sigma in S/m, absolute
    epsilon) and gradients with the reference's Tikhonov_cost_TE of a misfit
    (cost_k) and Tikhonov_grad_TE (gs_k, ge_k); case_k = (nx, ny, dh, IDX,
    IDY, MAT1_NORM, MAT2_NORM, BETA_MAT1, BETA_MAT2, LAMBDA_1, LAMBDA_2, L2)."""
    rng = np.random.default_rng(29)
    d = {"ncases": len(TIKH_CASES)}
    for k, (nx, ny, dh, idx, idy, n1, n2, b1, b2, l1, l2) in enumerate(TIKH_CASES):
        g = O.Grid(nx=nx, ny=ny, dh=dh, npml=4)
        sig = rng.uniform(1e-4, 1e-2, (ny, nx)).astype(np.float32)
        eps = (rng.uniform(3, 25, (ny, nx)) * 8.8541878e-12).astype(np.float32)
        gsig = rng.standard_normal((ny, nx)).astype(np.float32)
        geps = rng.standard_normal((ny, nx)).astype(np.float32)
        misfit = np.float32(rng.uniform(1, 100))
        ref = O.Ref(g)
        cost = ref.tikhonov_cost_te(sig, eps, misfit, n1, n2, b1, b2, l1, l2, idx, idy)
        gs, ge = ref.tikhonov_grad_te(gsig, geps, sig, eps, n1, n2, b1, b2, l1, l2, idx, idy)
        d.update({f"case_{k}": np.array([nx, ny, dh, idx, idy, n1, n2, b1, b2, l1, l2, misfit]), f"sig_{k}": sig,
                  f"eps_{k}": eps, f"gsig_{k}": gsig, f"geps_{k}": geps, f"cost_{k}": np.float32(cost),
                  f"gs_{k}": gs, f"ge_{k}": ge})
    np.savez_compressed(os.path.join(out, "postproc_tikhonov_te.npz"), **d)
    print("wrote postproc_tikhonov_te")


# precond cases: grid nx, ny, npml, free_surf, SPATFILTER, SWS_TAPER_GRAD_HOR, GRADT2, taper file
PRECOND_CASES = [(41, 33, 5, 0, 0, 1, 3, False), (41, 33, 5, 0, 0, 0, 0, True), (38, 29, 4, 1, 0, 0, 0, True),
                 (45, 31, 6, 0, 1, 1, 4, True), (36, 30, 5, 1, 1, 1, 2, True)]


def precond_fixture(out):
    """postproc_precond.npz: per case k the grid / switches (case_k), a
    seeded gradient (grad_k), the taper file content (taper_k, NX0*NY0 x
    outer, or empty) and the reference's precond output (out_k); gauss_filt
    with VREF 2000, FC_low 5, sizes 0.3 / 0.5 where SPATFILTER = 1."""
    rng = np.random.default_rng(19)
    d = {"ncases": len(PRECOND_CASES)}
    with tempfile.TemporaryDirectory() as tmp:
        for k, (nx, ny, npml, fs, spat, hor, gt2, tfile) in enumerate(PRECOND_CASES):
            g = O.Grid(nx=nx, ny=ny, dh=10.0, npml=npml, free_surf=fs)
            nx0, ny0 = nx - 2 * npml, ny - npml - g.fsshift
            grad = rng.standard_normal((ny, nx)).astype(np.float32)
            taper = rng.uniform(0.0, 1.0, nx0 * ny0).astype(np.float32) if tfile else None
            o = O.Ref(g).precond(tmp, grad, spat, 2000.0, 5.0, 0.3, 0.5, hor, gt2, taper)
            d.update({f"case_{k}": np.array([nx, ny, npml, fs, spat, hor, gt2, int(tfile)]), f"grad_{k}": grad,
                      f"taper_{k}": taper if taper is not None else np.zeros(0, np.float32), f"out_{k}": o})
    np.savez_compressed(os.path.join(out, "postproc_precond.npz"), **d)
    print("wrote postproc_precond")


# file-format cases: grid nx, ny, npml, free_surf
FILE_GRIDS = [(30, 22, 5, 0), (27, 19, 4, 1)]


def files_fixture(out):
    """files_formats.npz: for each grid k, seeded inputs (seis_k: seismograms
    [nf][nshots][ntr]; grid_k: a full [NY][NX] float grid; vp_k, rho_k: the
    interiors of a material file pair, x outer) and the files the reference
    writes or the arrays it reads from them: seis_file_k (write_seis_AC),
    true_file_k and true2_file_k (writemod_true, IDX = IDY = 1 and IDX = 2,
    IDY = 3), full_file_k (writemod format 3), readmod_vp_k / readmod_rho_k
    (readmod)."""
    rng = np.random.default_rng(23)
    d = {"ngrids": len(FILE_GRIDS)}
    with tempfile.TemporaryDirectory() as tmp:
        def rd(f):
            with open(os.path.join(tmp, f), "rb") as fh:
                return np.frombuffer(fh.read(), np.uint8)
        for k, (nx, ny, npml, fs) in enumerate(FILE_GRIDS):
            g = O.Grid(nx=nx, ny=ny, dh=10.0, npml=npml, free_surf=fs)
            ref = O.Ref(g)
            nf, ns, ntr = 3, 4, nx - 2 * npml
            seis = (rng.standard_normal((nf, ns, ntr)) + 1j * rng.standard_normal((nf, ns, ntr))).astype(np.complex64)
            grid = rng.standard_normal((ny, nx)).astype(np.float32)
            nx0, ny0 = nx - 2 * npml, ny - npml - g.fsshift
            vp = rng.uniform(1500, 4500, (nx0, ny0)).astype(np.float32)
            rho = rng.uniform(1000, 2600, (nx0, ny0)).astype(np.float32)
            ref.write_seis(os.path.join(tmp, f"picks{k}"), 2, seis)
            ref.writemod_true(os.path.join(tmp, "t1"), grid)
            ref.writemod_true(os.path.join(tmp, "t2"), grid, 2, 3)
            ref.writemod(os.path.join(tmp, "f1"), grid)
            mfile = os.path.join(tmp, f"model{k}")
            vp.tofile(mfile + ".vp")
            rho.tofile(mfile + ".rho")
            rvp, rrho = ref.readmod(mfile)
            d.update({f"case_{k}": np.array([nx, ny, npml, fs]), f"seis_{k}": seis, f"grid_{k}": grid,
                      f"vp_{k}": vp, f"rho_{k}": rho, f"seis_file_{k}": rd(f"picks{k}_p_stage_2.bin"),
                      f"true_file_{k}": rd("t1"), f"true2_file_{k}": rd("t2"), f"full_file_{k}": rd("f1"),
                      f"readmod_vp_{k}": rvp, f"readmod_rho_{k}": rrho})
    np.savez_compressed(os.path.join(out, "files_formats.npz"), **d)
    print("wrote files_formats")


if __name__ == "__main__":
    main()
