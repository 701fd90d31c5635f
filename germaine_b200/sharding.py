"""Frequency sharding over ranks with one exchange step: the gradient sum
(FWI) or the seismogram gather (forward modelling).

The reference distributes the frequencies of a stage over MPI ranks
(``init_MPIfreq``, src/init_MPIfreq.c:20-31: contiguous blocks, the first
``NF % NPROCFREQ`` ranks one frequency more), lets every rank evaluate its
frequencies' misfit and gradient independently (src/AC/grad_obj_AC.c:38-170)
and sums both over all ranks (``sum_grad_MPI``, src/sum_grad_MPI.c:36, and
the L2 ``MPI_Allreduce`` at grad_obj_AC.c:181) before the frame taper.

Here one rank drives one GPU: it factorises and solves only its own
frequencies (no data-path collective) and the partial gradients and misfits
are summed by ONE ``torch.distributed.all_reduce`` over a flat float64
buffer ``[grad0, grad1?, l2]`` -- NCCL over NVLink on GPUs, gloo on CPU
tests.  The taper (``cp_grad_frame``) is a per-cell factor, so tapering the
partial sums (what ``gm_grad_obj`` does) equals tapering the total.

Forward modelling (src/AC/forward_AC.c:155-173) exchanges the seismograms
once per stage in ``write_seis_AC`` (src/AC/write_seis_AC.c:33-45): every
rank holds the full [NF][nshots][ntr] arrays, zero outside its own
frequencies, and they are summed over all ranks.  Here each rank
contributes only its frequency block, in ONE ``all_gather``.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence, Tuple

import numpy as np

from ._lib import GM_PHYS_TE

__all__ = ["frequency_range", "local_frequencies", "allreduce_gradient", "sharded_grad_obj", "engine_grad_obj",
           "gather_seismograms", "sharded_forward", "engine_forward"]


def frequency_range(nf: int, nproc: int, rank: int) -> Tuple[int, int]:
    """0-based half-open range [lo, hi) of the frequencies of `rank`
    (NFREQ1-1, NFREQ2-1 of init_MPIfreq, src/init_MPIfreq.c:20-31)."""
    if nproc <= 0 or not 0 <= rank < nproc:
        raise ValueError(f"rank {rank} out of range for {nproc} ranks")
    base, extra = divmod(nf, nproc)
    lo = base * rank + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def local_frequencies(freqs: Sequence[float], nproc: int, rank: int) -> list:
    lo, hi = frequency_range(len(freqs), nproc, rank)
    return list(freqs[lo:hi])


def allreduce_gradient(g0: np.ndarray, g1: Optional[np.ndarray], l2: float, dist, group=None,
                       device=None) -> Tuple[np.ndarray, Optional[np.ndarray], float]:
    """Sum (g0, g1, l2) over the ranks of `group` in one all-reduce.
    `device` is where the buffer lives for the collective (a CUDA device for
    NCCL, None for gloo on CPU)."""
    import torch
    n = g0.size
    parts = [np.asarray(g0, np.float64).ravel()]
    if g1 is not None:
        parts.append(np.asarray(g1, np.float64).ravel())
    parts.append(np.array([l2], np.float64))
    buf = torch.from_numpy(np.concatenate(parts))
    if device is not None:
        buf = buf.to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out = buf.cpu().numpy()
    r0 = out[:n].copy()
    r1 = out[n:2 * n].copy() if g1 is not None else None
    return r0, r1, float(out[-1])


def sharded_grad_obj(freqs: Sequence[float],
                     local_grad_obj: Callable[[list], Tuple[np.ndarray, Optional[np.ndarray], float]],
                     dist, group=None, device=None) -> Tuple[np.ndarray, Optional[np.ndarray], float]:
    """Misfit and FP64 gradient over all `freqs`, each rank evaluating only
    its init_MPIfreq share with `local_grad_obj(local_freqs) -> (g0, g1, l2)`
    (called with an empty list on a rank without frequencies, where it
    returns zeros), then summed over the ranks.  Every rank takes the same
    collective step, whatever its share."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    g0, g1, l2 = local_grad_obj(local_frequencies(freqs, world, rank))
    return allreduce_gradient(g0, g1, l2, dist, group=group, device=device)


def engine_grad_obj(engine, src_x, src_y, rec_x, rec_y, pobs_by_freq: dict, stf_inv: int = 0, misfit: int = 1):
    """`local_grad_obj` for :func:`sharded_grad_obj` over a GPU
    :class:`~germaine_b200.engine.Engine`: factorises the rank's frequencies,
    runs gm_grad_obj over all shots and returns the FP64 gradients.
    `pobs_by_freq[f]` is the [nshots][ntr] observed data of frequency f."""
    def run(local: list):
        if not local:
            g1 = np.zeros(engine.n) if engine.physics == GM_PHYS_TE else None
            return np.zeros(engine.n), g1, 0.0
        engine.factor(local)
        obs = np.stack([np.asarray(pobs_by_freq[f], np.complex64) for f in local])
        _, _, l2, _ = engine.grad_obj(src_x, src_y, rec_x, rec_y, obs, stf_inv=stf_inv, misfit=misfit)
        g0, g1 = engine.gradient_fp64()
        return g0, g1, l2
    return run


def gather_seismograms(local_seis, nf: int, nshots: int, ntr: int, dist, group=None, device=None) -> np.ndarray:
    """Seismograms of all `nf` frequencies, [nf][nshots][ntr] complex64, on
    every rank of `group`, from each rank's init_MPIfreq block `local_seis`
    ([hi - lo][nshots][ntr]; None or empty on a rank without frequencies).

    The reference sums zero-filled full arrays over the ranks
    (src/AC/write_seis_AC.c:33-45); every entry has one contributor, so the
    blocks put side by side hold the same values, except that the sum turns
    a -0.0 into +0.0 when more than one rank takes part, which the last
    step repeats.  One all_gather of the blocks as float32 pairs, each block
    padded to the largest share (init_MPIfreq shares differ by at most one
    frequency).  `device` is where the buffers live for the collective."""
    import torch
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = frequency_range(nf, world, rank)
    width = -(-nf // world)
    blk = np.zeros((width, nshots, ntr), np.complex64)
    if hi > lo:
        loc = np.asarray(local_seis, np.complex64)
        if loc.shape != (hi - lo, nshots, ntr):
            raise ValueError(f"rank {rank}: seismograms {loc.shape}, expected {(hi - lo, nshots, ntr)}")
        blk[:hi - lo] = loc
    t = torch.from_numpy(blk.view(np.float32))
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    out = np.empty((nf, nshots, ntr), np.complex64)
    for r, part in enumerate(parts):
        a, b = frequency_range(nf, world, r)
        out[a:b] = part.cpu().numpy().view(np.complex64)[:b - a]
    if world > 1:
        out += np.complex64(0)
    return out


def sharded_forward(freqs: Sequence[float], local_forward: Callable[[list], np.ndarray], nshots: int, ntr: int,
                    dist, group=None, device=None) -> np.ndarray:
    """Seismograms [nf][nshots][ntr] of all `freqs` on every rank, each rank
    modelling only its init_MPIfreq share with
    `local_forward(local_freqs) -> [len(local_freqs)][nshots][ntr]` (called
    with an empty list on a rank without frequencies), then gathered.  Every
    rank takes the same collective step, whatever its share."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    local = local_frequencies(freqs, world, rank)
    seis = local_forward(local)
    return gather_seismograms(seis, len(freqs), nshots, ntr, dist, group=group, device=device)


def engine_forward(engine, src_x, src_y, rec_x, rec_y):
    """`local_forward` for :func:`sharded_forward` over a GPU
    :class:`~germaine_b200.engine.Engine`: factorises the rank's frequencies
    and runs gm_forward over all shots."""
    def run(local: list):
        if not local:
            return None
        engine.factor(local)
        seis, _ = engine.forward(src_x, src_y, rec_x, rec_y)
        return seis
    return run
