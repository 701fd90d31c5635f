"""Frequency (and shot) sharding over ranks with one data exchange: the
gradient sum (FWI) or the seismogram gather (forward modelling).

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
entries, and they are summed over all ranks.  Here each rank contributes
only its block, in ONE ``all_gather``.

The reference can also split the shots of a frequency (NPROCSHOT > 1):
rank MYID takes the frequency block of MYID % NPROCFREQ and the shot block
of MYID / NPROCFREQ (src/AC/fwi_FD_AC.c:201-211, init_MPIshot at
src/init_MPIshot.c:20-31), factorising its frequencies redundantly with the
other ranks of its frequency block.  ``nprocfreq`` selects that layout
(default: every rank a frequency block of its own, all shots).

Failures: a rank whose local evaluation raises still takes every
collective step.  One small all-reduce of a failure count precedes the
exchange; the failing rank then re-raises its own exception and the others
raise :class:`RankFailure`, so no rank waits for a peer that will not come.
A rank that stalls or dies is caught by the process group's timeout.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence, Tuple

import numpy as np

from ._lib import GM_PHYS_TE

__all__ = ["RankFailure", "frequency_range", "shot_range", "rank_blocks", "local_frequencies", "allreduce_gradient",
           "sharded_grad_obj", "engine_grad_obj", "gather_seismograms", "sharded_forward", "engine_forward"]


class RankFailure(RuntimeError):
    """Another rank's local evaluation failed; raised on every rank that
    did not fail itself, after the failure-count step."""


def _failures(ok: bool, dist, group, device) -> int:
    """Number of ranks whose local evaluation failed: one all-reduce that
    every rank takes, failed or not."""
    import torch
    t = torch.tensor([0.0 if ok else 1.0], dtype=torch.float64)
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return int(t.item())


def _run_local(fn, args, dist, group, device):
    """fn(*args) on this rank, then the failure-count step."""
    try:
        res, err = fn(*args), None
    except Exception as ex:   # the exchange must still be taken
        res, err = None, ex
    failed = _failures(err is None, dist, group, device)
    if err is not None:
        raise err
    if failed:
        raise RankFailure(f"{failed} rank(s) failed their local evaluation")
    return res


def _block(count: int, parts: int, me: int) -> Tuple[int, int]:
    """0-based half-open block [lo, hi) of `count` items of part `me` of
    `parts`: the first count % parts parts one item more (init_MPIfreq,
    src/init_MPIfreq.c:20-31; init_MPIshot, src/init_MPIshot.c:20-31)."""
    if parts <= 0 or not 0 <= me < parts:
        raise ValueError(f"rank {me} out of range for {parts} ranks")
    base, extra = divmod(count, parts)
    lo = base * me + min(me, extra)
    return lo, lo + base + (1 if me < extra else 0)


def frequency_range(nf: int, nproc: int, rank: int) -> Tuple[int, int]:
    """0-based half-open range [lo, hi) of the frequencies of `rank`
    (NFREQ1-1, NFREQ2-1 of init_MPIfreq, src/init_MPIfreq.c:20-31)."""
    return _block(nf, nproc, rank)


def shot_range(nshots: int, nprocshot: int, color: int) -> Tuple[int, int]:
    """0-based half-open range [lo, hi) of the shots of colour `color`
    (NSHOT1-1, NSHOT2-1 of init_MPIshot, src/init_MPIshot.c:20-31)."""
    return _block(nshots, nprocshot, color)


def rank_blocks(nf: int, nshots: int, world: int, rank: int,
                nprocfreq: Optional[int] = None) -> Tuple[Tuple[int, int], Tuple[int, int]]:
    """(frequency range, shot range) of `rank` among `world` ranks in the
    reference's layout (src/AC/fwi_FD_AC.c:201-211): COLOR = rank /
    NPROCFREQ picks the shot block among NPROCSHOT = world / NPROCFREQ, the
    rank within its colour (rank % NPROCFREQ) the frequency block.
    `nprocfreq` None means NPROCFREQ = world (all shots on every rank);
    world must be a multiple of it."""
    npf = world if nprocfreq is None else nprocfreq
    if npf <= 0 or world % npf:
        raise ValueError(f"{world} ranks are not a multiple of NPROCFREQ = {npf}")
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for {world} ranks")
    return frequency_range(nf, npf, rank % npf), shot_range(nshots, world // npf, rank // npf)


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
                     local_grad_obj: Callable[[list, Optional[range]], Tuple[np.ndarray, Optional[np.ndarray], float]],
                     dist, group=None, device=None, nshots: Optional[int] = None,
                     nprocfreq: Optional[int] = None) -> Tuple[np.ndarray, Optional[np.ndarray], float]:
    """Misfit and FP64 gradient over all `freqs` and shots, each rank
    evaluating only its share with `local_grad_obj(local_freqs, shots) ->
    (g0, g1, l2)`, then summed over the ranks.  `shots` is the rank's range
    of shot indices, or None for all shots (NPROCSHOT = 1); a rank without
    frequencies or shots is still called (with an empty list or range) and
    returns zeros.  `nshots` is needed only with `nprocfreq`.  Every rank
    takes the same collective steps, whatever its share and whether or not
    its evaluation fails (see the module's notes on failures)."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    local, shots = _share(freqs, nshots, world, rank, nprocfreq)
    g0, g1, l2 = _run_local(local_grad_obj, (local, shots), dist, group, device)
    return allreduce_gradient(g0, g1, l2, dist, group=group, device=device)


def _share(freqs, nshots, world, rank, nprocfreq):
    if nprocfreq is None or nprocfreq == world:
        return local_frequencies(freqs, world, rank), None
    if nshots is None:
        raise ValueError("nshots is needed to split the shots (nprocfreq < world)")
    (flo, fhi), (slo, shi) = rank_blocks(len(freqs), nshots, world, rank, nprocfreq)
    return list(freqs[flo:fhi]), range(slo, shi)


def engine_grad_obj(engine, src_x, src_y, rec_x, rec_y, pobs_by_freq: dict, stf_inv: int = 0, misfit: int = 1):
    """`local_grad_obj` for :func:`sharded_grad_obj` over a GPU
    :class:`~germaine_b200.engine.Engine`: factorises the rank's frequencies,
    runs gm_grad_obj over the rank's shots and returns the FP64 gradients.
    `pobs_by_freq[f]` is the [nshots][ntr] observed data of frequency f."""
    def run(local: list, shots: Optional[range] = None):
        sel = slice(None) if shots is None else slice(shots.start, shots.stop)
        if not local or (shots is not None and len(shots) == 0):
            g1 = np.zeros(engine.n) if engine.physics == GM_PHYS_TE else None
            return np.zeros(engine.n), g1, 0.0
        engine.factor(local)
        obs = np.stack([np.asarray(pobs_by_freq[f], np.complex64)[sel] for f in local])
        _, _, l2, _ = engine.grad_obj(np.asarray(src_x)[sel], np.asarray(src_y)[sel], rec_x, rec_y, obs,
                                      stf_inv=stf_inv, misfit=misfit)
        g0, g1 = engine.gradient_fp64()
        return g0, g1, l2
    return run


def gather_seismograms(local_seis, nf: int, nshots: int, ntr: int, dist, group=None, device=None,
                       nprocfreq: Optional[int] = None) -> np.ndarray:
    """Seismograms of all `nf` frequencies and `nshots` shots, [nf][nshots][ntr]
    complex64, on every rank of `group`, from each rank's block `local_seis`
    ([its frequencies][its shots][ntr] in the layout of :func:`rank_blocks`;
    None or empty on a rank without frequencies or shots).

    The reference sums zero-filled full arrays over the ranks
    (src/AC/write_seis_AC.c:33-45); every entry has one contributor, so the
    blocks put side by side hold the same values, except that the sum turns
    a -0.0 into +0.0 when more than one rank takes part, which the last
    step repeats.  (Its sum starts one element early and so leaves the last
    sample 0; that is a property of the file it writes, which
    files.write_seis reproduces, not of the data.)  One all_gather of the blocks as float32 pairs, each block
    padded to the largest share (the shares differ by at most one frequency
    and one shot).  `device` is where the buffers live for the collective."""
    import torch
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    npf = world if nprocfreq is None else nprocfreq
    (flo, fhi), (slo, shi) = rank_blocks(nf, nshots, world, rank, npf)
    fw, sw = -(-nf // npf), -(-nshots // (world // npf))
    blk = np.zeros((fw, sw, ntr), np.complex64)
    if fhi > flo and shi > slo:
        loc = np.asarray(local_seis, np.complex64)
        if loc.shape != (fhi - flo, shi - slo, ntr):
            raise ValueError(f"rank {rank}: seismograms {loc.shape}, expected {(fhi - flo, shi - slo, ntr)}")
        blk[:fhi - flo, :shi - slo] = loc
    t = torch.from_numpy(blk.view(np.float32))
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    out = np.empty((nf, nshots, ntr), np.complex64)
    for r, part in enumerate(parts):
        (a, b), (c, d) = rank_blocks(nf, nshots, world, r, npf)
        out[a:b, c:d] = part.cpu().numpy().view(np.complex64)[:b - a, :d - c]
    if world > 1:
        out += np.complex64(0)
    return out


def sharded_forward(freqs: Sequence[float], local_forward: Callable[[list, Optional[range]], np.ndarray],
                    nshots: int, ntr: int, dist, group=None, device=None,
                    nprocfreq: Optional[int] = None) -> np.ndarray:
    """Seismograms [nf][nshots][ntr] of all `freqs` and shots on every rank,
    each rank modelling only its share with `local_forward(local_freqs,
    shots) -> [len(local_freqs)][len(shots)][ntr]` (`shots` None = all
    shots; called with an empty list or range on a rank without work), then
    gathered.  Every rank takes the same collective steps, whatever its
    share and whether or not its evaluation fails."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    local, shots = _share(freqs, nshots, world, rank, nprocfreq)
    (flo, fhi), (slo, shi) = rank_blocks(len(freqs), nshots, world, rank, nprocfreq)

    def checked(local, shots):   # a block of the wrong shape fails before the exchange, like any other error
        seis = local_forward(local, shots)
        if fhi > flo and shi > slo and np.shape(seis) != (fhi - flo, shi - slo, ntr):
            raise ValueError(f"rank {rank}: seismograms {np.shape(seis)}, expected {(fhi - flo, shi - slo, ntr)}")
        return seis
    seis = _run_local(checked, (local, shots), dist, group, device)
    return gather_seismograms(seis, len(freqs), nshots, ntr, dist, group=group, device=device,
                              nprocfreq=nprocfreq)


def engine_forward(engine, src_x, src_y, rec_x, rec_y):
    """`local_forward` for :func:`sharded_forward` over a GPU
    :class:`~germaine_b200.engine.Engine`: factorises the rank's frequencies
    and runs gm_forward over the rank's shots."""
    def run(local: list, shots: Optional[range] = None):
        if not local or (shots is not None and len(shots) == 0):
            return None
        sel = slice(None) if shots is None else slice(shots.start, shots.stop)
        engine.factor(local)
        seis, _ = engine.forward(np.asarray(src_x)[sel], np.asarray(src_y)[sel], rec_x, rec_y)
        return seis
    return run
