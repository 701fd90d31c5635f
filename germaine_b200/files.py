"""The reference's on-disk formats through the C-ABI (gm_write_seis,
gm_read_seis, gm_write_model_true, gm_write_model, gm_read_model), so that
seismograms and models move between this engine and GERMAINE unchanged:

* seismograms ``<PICKS_FILE>_p_stage_<n>.bin`` of write_seis_AC
  (src/AC/write_seis_AC.c:53-67), read by read_seis_AC
  (src/AC/read_seis_AC.c:24-37): complex64 [NF][NSHOTS][NTR].  The
  reference's writer always stores the file's last sample as 0 + 0i (its
  gather at src/AC/write_seis_AC.c:43-44 starts one element early);
  ``write_seis`` does the same unless ``keep_last=True``;
* models and snapshots without the PML frame, writemod_true
  (src/writemod_true.c:26-34), and with it, writemod format 3
  (src/writemod.c:24-30);
* material files ``<MFILE>.vp`` / ``.rho`` (``.vs``, ``.sig``, ``.eps``)
  of readmod (src/readmod.c:43-104), extended into the PML frame.
"""
import os

import numpy as np

from . import _lib
from ._lib import check, ptr


def _path(path) -> bytes:
    return os.fsencode(path)


def seis_path(prefix: str, stage: int) -> str:
    """File name write_seis_AC builds from PICKS_FILE and the stage
    (src/AC/write_seis_AC.c:50)."""
    return f"{prefix}_p_stage_{stage}.bin"


def write_seis(path, seis, keep_last: bool = False) -> None:
    """Write complex64 seismograms [nf][nshots][ntr] as write_seis_AC does
    (last sample zero, byte-identical), or with every sample kept."""
    s = np.ascontiguousarray(seis, np.complex64)
    if s.ndim != 3:
        raise ValueError("seismograms must be [nf][nshots][ntr]")
    flags = _lib.GM_SEIS_KEEP_LAST if keep_last else 0
    check(_lib.load().gm_write_seis(_path(path), *s.shape, flags, ptr(s)))


def read_seis(path, nf: int, nshots: int, ntr: int) -> np.ndarray:
    """Read observed seismograms as read_seis_AC does."""
    s = np.empty((nf, nshots, ntr), np.complex64)
    check(_lib.load().gm_read_seis(_path(path), nf, nshots, ntr, ptr(s)))
    return s


def write_model_true(path, grid, npml: int, free_surf: int = 0, idx: int = 1, idy: int = 1) -> None:
    """Write the interior of a [NY][NX] grid as writemod_true does."""
    g = np.ascontiguousarray(grid, np.float32)
    ny, nx = g.shape
    check(_lib.load().gm_write_model_true(_path(path), nx, ny, npml, free_surf, idx, idy, ptr(g)))


def write_model(path, grid, idx: int = 1, idy: int = 1) -> None:
    """Write a full [NY][NX] grid as writemod (binary format 3) does."""
    g = np.ascontiguousarray(grid, np.float32)
    ny, nx = g.shape
    check(_lib.load().gm_write_model(_path(path), nx, ny, idx, idy, ptr(g)))


def read_grid(path, nx: int, ny: int) -> np.ndarray:
    """Read a full [NY][NX] grid written x outer (writemod format 3, the
    reference's l-BFGS "*.old" and Hessian files)."""
    g = np.empty((ny, nx), np.float32)
    check(_lib.load().gm_read_grid(_path(path), nx, ny, ptr(g)))
    return g


def read_model(path, nx: int, ny: int, npml: int, free_surf: int = 0) -> np.ndarray:
    """Read one material file into a [NY][NX] grid (NX, NY include the PML
    frame) and extend it into the frame as readmod does."""
    g = np.empty((ny, nx), np.float32)
    check(_lib.load().gm_read_model(_path(path), nx, ny, npml, free_surf, ptr(g)))
    return g
