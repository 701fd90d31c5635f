"""Generates tests/golden/*.npz from the reference's OWN sources (compiled
into oracle/_ref by `make -C oracle ref`, where the reference tree is
present).  Each fixture holds one small seeded model, the reference's PML
profiles and assembled triplets (init_A_*_9p_pml) and, for the acoustic
cases, a right-hand side with its FP64 sparse solution on the operator
UMFPACK factorises (M = A^T; solved with SciPy SuperLU because UMFPACK is
not part of the reference tree).  Run:  python tests/golden/make_golden.py
"""
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
    gauss_filt_fixture(out)


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


if __name__ == "__main__":
    main()
