"""Seeded synthetic workloads with the shapes and value ranges of the
benchmark configurations (the reference's own example models come from an
external benchmark collection that is not part of the reference tree).

* ``thrust_model``   -- folded / thrust-faulted layered acoustic model:
  8-12 sinusoidal-plus-step interfaces, vp 2360-6000 m/s increasing with
  depth, constant density; interior NX0 x NY0 at spacing DH, extended into
  the PML frame the way readmod() does (src/readmod.c:60-92).
* ``inclusion_model`` -- homogeneous 2000 m/s / 1000 kg/m^3 with one circular
  2400 m/s inclusion of radius 150 m at the centre.
* ``gpr_model``      -- georadar (TE) model: layered relative permittivity
  3-25 with elliptical anomalies, conductivity 0.1-10 mS/m.
* ``line_acquisition`` -- shots and receivers along one model row.
"""
from __future__ import annotations

import numpy as np


def extend_into_pml(a_int: np.ndarray, npml: int, free_surf: int = 0) -> np.ndarray:
    """Pad an interior [NY0][NX0] model with the PML frame by edge copies."""
    top = 0 if free_surf else npml
    return np.pad(a_int, ((top, npml), (npml, npml)), mode="edge").astype(np.float32)


def thrust_model(nx0: int = 801, ny0: int = 187, dh: float = 25.0, npml: int = 20, seed: int = 2024,
                 rho: float = 1000.0):
    rng = np.random.default_rng(seed)
    nif = int(rng.integers(8, 13))
    x = np.arange(nx0) * dh
    depth = ny0 * dh
    base = np.sort(rng.uniform(0.08, 0.95, nif)) * depth
    z = np.empty((nif, nx0))
    for i in range(nif):
        amp = rng.uniform(0.01, 0.06) * depth
        lam = rng.uniform(0.3, 1.2) * x[-1]
        phase = rng.uniform(0, 2 * np.pi)
        xs = rng.uniform(0.2, 0.8) * x[-1]                    # thrust position
        step = rng.uniform(-0.05, 0.05) * depth               # fault throw
        ramp = 0.5 * (1 + np.tanh((x - xs) / (3 * dh)))
        z[i] = base[i] + amp * np.sin(2 * np.pi * x / lam + phase) + step * ramp
    z = np.maximum.accumulate(np.sort(z, axis=0), axis=0)      # interfaces do not cross
    vel = np.sort(rng.uniform(2360.0, 6000.0, nif + 1))
    vel[0], vel[-1] = 2360.0, 6000.0
    yy = (np.arange(ny0) * dh)[:, None]
    layer = np.zeros((ny0, nx0), np.int64)
    for i in range(nif):
        layer += (yy >= z[i][None, :]).astype(np.int64)
    vp = vel[layer].astype(np.float32)
    vp_full = extend_into_pml(vp, npml)
    return vp_full, np.full_like(vp_full, rho)


def inclusion_model(nx0: int = 201, ny0: int = 101, dh: float = 10.0, npml: int = 20, v0: float = 2000.0,
                    v1: float = 2400.0, rho: float = 1000.0, radius: float = 150.0):
    x = (np.arange(nx0) + 0.5) * dh
    y = (np.arange(ny0) + 0.5) * dh
    X, Y = np.meshgrid(x, y)
    vp = np.full((ny0, nx0), v0, np.float32)
    vp[(X - nx0 * dh / 2) ** 2 + (Y - ny0 * dh / 2) ** 2 <= radius ** 2] = v1
    vp_full = extend_into_pml(vp, npml)
    return vp_full, np.full_like(vp_full, rho)


def gpr_model(nx0: int = 4000, ny0: int = 2000, dh: float = 0.025, npml: int = 30, seed: int = 2025,
              nlayers: int = 6, nellipses: int = 12):
    """Georadar (TE) model: seeded random layers of relative permittivity
    3-25 with elliptical anomalies, conductivity 0.1-10 mS/m; returns the
    absolute permittivity (eps_r * eps0, F/m) and the conductivity (S/m),
    [NY][NX] with the PML frame."""
    eps0 = 8.854187817e-12
    rng = np.random.default_rng(seed)
    x = (np.arange(nx0) * dh)[None, :]
    y = (np.arange(ny0) * dh)[:, None]
    depth = ny0 * dh
    tops = np.sort(rng.uniform(0.05, 0.95, nlayers - 1)) * depth
    eps = np.full((ny0, nx0), rng.uniform(3.0, 25.0), np.float64)
    sig = np.full((ny0, nx0), 10 ** rng.uniform(-4.0, -2.0), np.float64)
    for t in tops:
        amp = rng.uniform(0.0, 0.03) * depth
        lam = rng.uniform(0.3, 1.0) * nx0 * dh
        surf = t + amp * np.sin(2 * np.pi * x / lam + rng.uniform(0, 2 * np.pi))
        below = y >= surf
        eps = np.where(below, rng.uniform(3.0, 25.0), eps)
        sig = np.where(below, 10 ** rng.uniform(-4.0, -2.0), sig)
    for _ in range(nellipses):
        cx, cy = rng.uniform(0.1, 0.9) * nx0 * dh, rng.uniform(0.1, 0.9) * depth
        ax, ay = rng.uniform(0.01, 0.08) * nx0 * dh, rng.uniform(0.01, 0.08) * depth
        inside = ((x - cx) / ax) ** 2 + ((y - cy) / ay) ** 2 <= 1.0
        eps = np.where(inside, rng.uniform(3.0, 25.0), eps)
        sig = np.where(inside, 10 ** rng.uniform(-4.0, -2.0), sig)
    eps_full = extend_into_pml((eps * eps0).astype(np.float32), npml)
    sig_full = extend_into_pml(sig.astype(np.float32), npml)
    return eps_full, sig_full


def line_acquisition(nx0: int, dh: float, nshots: int, row: int, nrec: int | None = None):
    """nshots sources evenly spaced along model row `row` (metres) and nrec
    receivers (default: every interior grid point) on the same row (grid
    indices without the PML offset, as recpos[1]/[2])."""
    xs = np.linspace(dh, (nx0 - 2) * dh, nshots).astype(np.float32)
    ys = np.full(nshots, row * dh, np.float32)
    if nrec is None:
        rx = np.arange(1, nx0, dtype=np.int32)
    else:
        rx = np.round(np.linspace(1, nx0 - 1, nrec)).astype(np.int32)
    ry = np.full(rx.size, row, np.int32)
    return xs, ys, rx, ry
