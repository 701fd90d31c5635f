"""Many frequencies, each on its own grid (the batched multi-grid workload):
a frequency's grid spacing follows from the shortest wavelength it must
resolve (h = vmin / (points_per_wavelength * f)), so every frequency of a
broadband inversion gets a grid of its own and the grids are uneven.  The
reference runs one frequency after another (forward_AC.c:155-169).

Here every grid gets an engine of its own (its symbolic analysis, its
fronts, its CUDA stream) and the engines run concurrently from host threads
(the C-ABI calls release the interpreter lock), so the tree levels of the
small grids' factorisations and substitutions run beside the large ones'
on the GPU instead of after them.
"""
from __future__ import annotations

import math
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from ._lib import GM_REFINE_MODE_IR
from .engine import Engine
from .synthetic import extend_into_pml


@dataclass
class GridCase:
    freq: float
    dh: float
    nx0: int
    ny0: int
    npml: int

    @property
    def shape(self):
        return self.ny0 + 2 * self.npml, self.nx0 + 2 * self.npml


def grids_for(freqs, extent_x: float, extent_y: float, vmin: float = 1500.0, ppw: float = 5.0, npml: int = 20,
              min_cells=(400, 100)):
    """One grid per frequency at ppw points per minimum wavelength, at least
    min_cells cells (the low frequencies keep that minimum, finer than their
    wavelength needs)."""
    out = []
    for f in freqs:
        dh = min(vmin / (ppw * f), extent_x / min_cells[0], extent_y / min_cells[1])
        out.append(GridCase(float(f), float(dh), int(math.ceil(extent_x / dh - 1e-9)),
                            int(math.ceil(extent_y / dh - 1e-9)), npml))
    return out


def c3_cases(nfreq: int = 32, fmin: float = 2.0, fmax: float = 17.0):
    """The batched multi-grid configuration: 32 frequencies in 2-17 Hz at 5
    points per minimum wavelength (vmin 1500 m/s), grids from 400 x 100 to
    1600 x 400 cells (+ a 20-point PML)."""
    dh_max = 1500.0 / (5.0 * fmax)
    return grids_for(np.linspace(fmin, fmax, nfreq), 1600 * dh_max, 400 * dh_max)


def smooth_random_model(extent_x: float, extent_y: float, dh: float, nx0: int, ny0: int, npml: int, seed: int,
                        vmin: float = 1500.0, vmax: float = 4500.0, corr: float = 400.0):
    """A seeded smooth Gaussian-perturbed velocity v(x, z) in [vmin, vmax]
    sampled on the grid (the same continuous model for every grid: its
    Fourier coefficients are drawn once from the seed), constant density."""
    rng = np.random.default_rng(seed)
    k = 24
    kx = rng.normal(0.0, 1.0 / corr, k)
    kz = rng.normal(0.0, 1.0 / corr, k)
    ph = rng.uniform(0, 2 * np.pi, k)
    amp = rng.normal(0.0, 1.0, k)
    x = (np.arange(nx0) + 0.5) * dh
    z = (np.arange(ny0) + 0.5) * dh
    X, Z = np.meshgrid(x, z)
    field = np.zeros_like(X)
    for i in range(k):
        field += amp[i] * np.cos(2 * np.pi * (kx[i] * X + kz[i] * Z) + ph[i])
    field = (field - field.min()) / max(field.max() - field.min(), 1e-12)
    depth_trend = Z / extent_y
    v = vmin + (vmax - vmin) * np.clip(0.6 * depth_trend + 0.4 * field, 0.0, 1.0)
    vp = extend_into_pml(v.astype(np.float32), npml)
    return vp, np.full_like(vp, 1000.0)


def run_multigrid(cases, nshots: int, seed: int = 7, precision: int = 1, workers: int | None = None,
                  row: int = 2, refine: int = 0, ir_max_iter: int = 30):
    """Factorise and solve every grid's frequency for nshots shots along
    model row `row`, all grids concurrently.  Returns (shot-solves/s over
    the whole set, wall seconds, per-grid records).

    refine defaults to the engine's automatic choice (plain sweeps, GMRES-IR
    for a grid whose sweeps contract too slowly: at 5 points per wavelength
    the complex64 factors of the highest frequencies stall plain sweeps).
    Two untimed passes place the buffers: the first, with plain sweeps
    only, allocates every grid's fronts and solve workspaces; the second,
    with the requested refinement, runs the grids one after another,
    smallest first, so that GMRES-IR sizes its Krylov vectors from the
    device memory all the grids leave.  The timed pass then runs every grid
    concurrently on the resident buffers.  ir_max_iter bounds the sweeps
    and GMRES iterations per grid (the highest-frequency grids need more
    than the default 10)."""
    extent_x = max(c.nx0 * c.dh for c in cases)
    extent_y = max(c.ny0 * c.dh for c in cases)
    engines, setups = [], []
    for c in cases:
        ny, nx = c.shape
        vp, rho = smooth_random_model(extent_x, extent_y, c.dh, c.nx0, c.ny0, c.npml, seed)
        xs = np.linspace(2 * c.dh, (c.nx0 - 3) * c.dh, nshots).astype(np.float32)
        ys = np.full(nshots, row * c.dh, np.float32)
        rx = np.arange(1, c.nx0, max(1, c.nx0 // 200), dtype=np.int32)
        ry = np.full(rx.size, row, np.int32)
        e = Engine(nx, ny, c.dh, c.npml, precision=precision, refine=GM_REFINE_MODE_IR, ir_max_iter=ir_max_iter)
        e.set_model(vp, rho)
        engines.append(e)
        setups.append((xs, ys, rx, ry))

    def one(i):
        e = engines[i]
        xs, ys, rx, ry = setups[i]
        e.factor([cases[i].freq])
        e.forward(xs, ys, rx, ry)
        st = e.stats()
        return {"freq": cases[i].freq, "grid": list(cases[i].shape), "n": st["n"], "ir_residual": st["ir_residual"],
                "status": e.last_status, "refine": e.refine_report()[0]}

    import torch
    try:
        with ThreadPoolExecutor(max_workers=workers or len(cases)) as pool:
            list(pool.map(one, range(len(cases))))              # fronts and solve workspaces
            torch.cuda.synchronize()
            for i in sorted(range(len(cases)), key=lambda i: engines[i].n):   # Krylov workspaces
                engines[i].set_refine(refine)
                one(i)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            recs = list(pool.map(one, range(len(cases))))
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
    finally:
        for e in engines:
            e.close()
    return len(cases) * nshots / wall, wall, recs
