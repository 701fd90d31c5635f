"""The mid-level kernel's 32-pivot form (fronts with 17-32 pivots, pivot rows
of 32 entries in registers).  By default such levels take the blocked
diagonal / panel / contribution-GEMM sequence, which measured faster;
GM_MID_MAX_PIV=32 routes them back to the fused kernel.  The variable is
read once per process, so the solve runs in a child process: the level
trace must show a "mid" level with more than 16 pivots, and the FP64
solution must match SuperLU (both orientations)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
import oracle as O
from oracle import sparse as OS
from germaine_b200 import GM_SYS_A, GM_SYS_AT, Engine
from tests.models import inclusion_ac, random_smooth
nx, ny, dh, npml = 241, 141, 10.0, 10
g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
vp, rho = inclusion_ac(nx, ny, dh, npml)
vp = vp * random_smooth(nx, ny, 0.85, 1.15, 9)
rng = np.random.default_rng(2)
b = rng.standard_normal((g.n, 3)) + 1j * rng.standard_normal((g.n, 3))
out = {}
with Engine(nx, ny, dh, npml) as e:
    e.set_model(vp, rho)
    e.factor([15.0])
    for name, sys_ in (("A", GM_SYS_A), ("At", GM_SYS_AT)):
        x = e.solve(b, sys_)
        M = OS.operator(OS.assembled_matrix(g, *e.triplets(0)), 0)
        xr = OS.DirectSolver(M).solve(b, trans=sys_ == GM_SYS_AT)
        out[name] = float(np.linalg.norm(x - xr) / np.linalg.norm(xr))
print(json.dumps(out))
"""


def test_mid_kernel_32_pivot_form_matches_superlu():
    env = dict(os.environ, GM_MID_MAX_PIV="32", GM_TRACE_LEVELS="1", PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    wide_mid = [ln for ln in r.stderr.splitlines()
                if ln.startswith("factor c128") and ln.split()[-3] == "mid" and int(ln.split()[9]) > 16]
    assert wide_mid, r.stderr[-2000:]
    errs = json.loads(r.stdout.strip().splitlines()[-1])
    assert errs["A"] < 1e-10 and errs["At"] < 1e-10, errs
