"""The large georadar configuration (C5): TE mode on 4000 x 2000 cells at
2.5 cm with a 30-point PML (4060 x 2060, 8.36 M unknowns), frequencies in
100-400 MHz, 500 transmitters along the surface.  The reference solves it
one frequency and one shot at a time (forward_shot_TE,
src/TE/forward_shot_TE.c:41-120); here one frequency's factors (53 GB in
FP64) stay resident and the shots are solved in blocks chosen by the
memory plan.  Checks: the FP64 and mixed-precision paths meet the residual
target on every frequency and agree on every seismogram; block solves give
the seismograms of one big solve; the wavefields of a 16-shot subset agree
to the mixed path's tolerance."""
import numpy as np
import pytest

from germaine_b200 import GM_PHYS_TE, GM_PREC_C64_IR, GM_PREC_FP64, Engine
from germaine_b200.synthetic import gpr_model

pytestmark = pytest.mark.gpu

NX0, NY0, DH, NPML = 4000, 2000, 0.025, 30
FREQS = [float(f) for f in np.linspace(100e6, 400e6, 16)]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def c5():
    eps, sig = gpr_model(NX0, NY0, DH, NPML, seed=2025)
    xs = np.linspace(2 * DH, (NX0 - 3) * DH, 500).astype(np.float32)
    ys = np.full(xs.size, 2 * DH, np.float32)
    rx = np.arange(1, NX0, 8, dtype=np.int32)           # 500 receivers along the surface
    ry = np.full(rx.size, 2, np.int32)
    return eps, sig, xs, ys, rx, ry


def test_c5_memory_plan_and_paths_agree(c5):
    import torch
    eps, sig, xs, ys, rx, ry = c5
    nx, ny = NX0 + 2 * NPML, NY0 + 2 * NPML
    free, _ = torch.cuda.mem_get_info()
    sub = [FREQS[0], FREQS[-1]]                          # the lowest and highest frequency
    seis = {}
    for prec in (GM_PREC_FP64, GM_PREC_C64_IR):
        with Engine(nx, ny, DH, NPML, physics=GM_PHYS_TE, precision=prec) as e:
            assert e.stats()["n"] == 8_363_600
            e.set_model(eps, sig)
            nfb, nsb = e.plan(len(FREQS), len(xs), int(0.8 * free))
            assert 1 <= nfb and 1 <= nsb <= len(xs)
            out = []
            for f in sub:
                e.factor([f])
                s, _ = e.forward(xs, ys, rx, ry)
                rep = e.refine_report()
                assert rep[0]["final_residual"] <= 1e-10, (prec, f, rep)
                out.append(s[0])
            seis[prec] = np.stack(out)
            if prec == GM_PREC_FP64:
                # blocks of 128 shots give the seismograms of the planned solve
                e.set_shot_block(128)
                e.factor(sub[:1])
                s128, _ = e.forward(xs, ys, rx, ry)
                assert _rel(s128[0], seis[prec][0]) < 1e-6
                e.set_shot_block(0)
    for i, f in enumerate(sub):
        assert _rel(seis[GM_PREC_C64_IR][i], seis[GM_PREC_FP64][i]) < 1e-6, f


def test_c5_wavefields_mixed_vs_fp64(c5):
    eps, sig, xs, ys, rx, ry = c5
    nx, ny = NX0 + 2 * NPML, NY0 + 2 * NPML
    xs16, ys16 = xs[::32][:16], ys[::32][:16]
    x = {}
    for prec in (GM_PREC_FP64, GM_PREC_C64_IR):
        with Engine(nx, ny, DH, NPML, physics=GM_PHYS_TE, precision=prec) as e:
            e.set_model(eps, sig)
            e.factor([FREQS[7]])
            e.forward(xs16, ys16, rx, ry)
            assert e.stats()["ir_residual"] <= 1e-10
            x[prec] = e.wavefield_fp64(0, len(xs16))
    assert _rel(x[GM_PREC_C64_IR], x[GM_PREC_FP64]) < 1e-8
