"""K1 assembly on the GPU vs the reference's own init_A_*_9p_pml (compiled
into oracle/_ref) and the C restatement: bit-identical triplets."""
import numpy as np
import pytest

import oracle as O
from germaine_b200 import GM_PHYS_AC, GM_PHYS_SH, GM_PHYS_TE, Engine
from tests.models import inclusion_ac, random_smooth, te_model

pytestmark = pytest.mark.gpu

CASES = [
    # physics, nx, ny, dh, npml, free_surf, s, freqs
    (GM_PHYS_AC, 61, 41, 10.0, 10, 0, 0.0, [15.0, 3.5]),
    (GM_PHYS_AC, 47, 33, 25.0, 8, 1, 1.7, [2.0, 11.0]),
    (GM_PHYS_SH, 53, 37, 10.0, 10, 0, 0.0, [9.0]),
    (GM_PHYS_SH, 40, 30, 12.5, 6, 0, 0.9, [4.0, 21.0]),
    (GM_PHYS_TE, 50, 44, 0.025, 10, 0, 0.0, [1e8, 4e8]),
    (GM_PHYS_TE, 36, 28, 0.05, 5, 1, 3e6, [2.5e8]),
]


def _model(physics, nx, ny, dh, npml, seed):
    if physics == GM_PHYS_AC:
        vp, rho = inclusion_ac(nx, ny, dh, npml)
        return vp * random_smooth(nx, ny, 0.9, 1.1, seed), rho * random_smooth(nx, ny, 0.8, 1.2, seed + 7)
    if physics == GM_PHYS_SH:
        return random_smooth(nx, ny, 800.0, 2500.0, seed), random_smooth(nx, ny, 1500.0, 2600.0, seed + 3)
    return te_model(nx, ny, seed)


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.uint64), np.asarray(b, np.float64).view(np.uint64))


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"phys{c[0]}-{c[1]}x{c[2]}-fs{c[5]}-S{c[6]}")
def test_assembly_bit_exact(case):
    physics, nx, ny, dh, npml, fs, s, freqs = case
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml, free_surf=fs, s=s)
    m0, m1 = _model(physics, nx, ny, dh, npml, seed=nx + ny)
    with Engine(nx, ny, dh, npml, physics=physics, free_surf=fs, s=s) as e:
        e.set_model(m0, m1)
        e.factor(freqs)
        ref = O.Ref(g) if O.ref_available() else None
        port = O.Port(g)
        for i, f in enumerate(freqs):
            ar, ai, ir, ic = e.triplets(i)
            pr = port.assemble(physics, f, m0, m1)
            assert np.array_equal(ir, pr[2]) and np.array_equal(ic, pr[3])
            assert _bits_equal(ar, pr[0]), f"real parts differ at {np.nonzero(ar != pr[0])[0][:5]}"
            assert _bits_equal(ai, pr[1]), f"imag parts differ at {np.nonzero(ai != pr[1])[0][:5]}"
            if ref is not None:
                rr = ref.assemble(physics, f, m0, m1)
                assert _bits_equal(ar, rr[0]) and _bits_equal(ai, rr[1])
