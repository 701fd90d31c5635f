"""Seeded synthetic models and acquisitions for the tests (shared helpers).

The reference's example models (DENISE-Benchmark inclusion / overthrust
files) are not part of the reference tree; these generators stand in for
them with the shapes and value ranges of the benchmark configurations.
"""
from __future__ import annotations

import numpy as np


def inclusion_ac(nx, ny, dh, npml, v0=2000.0, v1=2400.0, rho=1000.0, radius=150.0):
    """Homogeneous model with one circular inclusion at the centre of the
    interior (the 201 x 101, 10 m benchmark case scaled to the grid),
    extended into the PML frame like readmod() does."""
    x = (np.arange(nx) - npml + 0.5) * dh
    y = (np.arange(ny) - npml + 0.5) * dh
    X, Y = np.meshgrid(x, y)
    cx, cy = (nx - 2 * npml) * dh / 2, (ny - 2 * npml) * dh / 2
    vp = np.full((ny, nx), v0, np.float32)
    vp[(X - cx) ** 2 + (Y - cy) ** 2 <= radius ** 2] = v1
    return vp, np.full((ny, nx), rho, np.float32)


def random_smooth(nx, ny, lo, hi, seed, corr=4.0):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    a = gaussian_filter(rng.standard_normal((ny, nx)), corr, mode="reflect")
    a = (a - a.min()) / max(a.max() - a.min(), 1e-12)
    return (lo + (hi - lo) * a).astype(np.float32)


def te_model(nx, ny, seed):
    eps0 = 8.854187817e-12
    epsr = random_smooth(nx, ny, 3.0, 25.0, seed)
    sig = random_smooth(nx, ny, 1e-4, 1e-2, seed + 1)
    return (epsr * eps0).astype(np.float32), sig


def line_shots(nx, npml, dh, ns, row=3):
    """ns sources evenly along model row `row` (positions in metres)."""
    nx0 = nx - 2 * npml
    xs = np.linspace(2 * dh, (nx0 - 3) * dh, ns).astype(np.float32)
    ys = np.full(ns, row * dh, np.float32)
    return xs, ys


def line_receivers(nx, npml, row=3, step=1):
    nx0 = nx - 2 * npml
    rx = np.arange(1, nx0 - 1, step, dtype=np.int32)
    ry = np.full(rx.size, row, np.int32)
    return rx, ry
