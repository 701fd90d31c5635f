"""Frequency sharding with one gradient all-reduce or one seismogram gather
(germaine_b200/sharding.py): the rank shares follow init_MPIfreq
(src/init_MPIfreq.c:20-31), the sharded misfit / FP64 gradient over gloo
ranks on CPU equals the single-process result, and the gathered
seismograms equal write_seis_AC's sum of zero-filled arrays
(src/AC/write_seis_AC.c:33-45) and the single-process forward.  The per-rank evaluation in the CPU tests is the FP64
oracle (SuperLU + FP64 restatements); on the GPU it is the engine, with the
all-reduce over NCCL."""
import os
import socket
import tempfile

import numpy as np
import pytest

from germaine_b200.sharding import (frequency_range, gather_seismograms, local_frequencies, rank_blocks,
                                    sharded_forward, sharded_grad_obj)


def init_mpifreq(nf, nprocfreq, myid_shot):
    """NFREQ1, NFREQ2 (1-based, half-open) as src/init_MPIfreq.c:20-31 computes them."""
    nfreq1 = (nf // nprocfreq) * myid_shot
    if nf % nprocfreq > myid_shot:
        nfreq1 += myid_shot
        nfreq2 = nfreq1 + nf // nprocfreq + 1
    else:
        nfreq1 += nf % nprocfreq
        nfreq2 = nfreq1 + nf // nprocfreq
    return nfreq1 + 1, nfreq2 + 1


@pytest.mark.parametrize("nf", [1, 2, 3, 7, 10, 16, 32])
@pytest.mark.parametrize("nproc", [1, 2, 3, 4, 8])
def test_frequency_range_is_init_mpifreq(nf, nproc):
    seen = []
    for rank in range(nproc):
        lo, hi = frequency_range(nf, nproc, rank)
        n1, n2 = init_mpifreq(nf, nproc, rank)
        assert (lo, hi) == (n1 - 1, n2 - 1)
        seen += list(range(lo, hi))
    assert seen == list(range(nf))


def test_frequency_range_rejects_bad_rank():
    with pytest.raises(ValueError):
        frequency_range(4, 2, 2)


def init_mpishot(nshots, nprocshot, color):
    """NSHOT1, NSHOT2 (1-based, half-open) as src/init_MPIshot.c:20-31 computes them."""
    nshot1 = (nshots // nprocshot) * color
    if nshots % nprocshot > color:
        nshot1 += color
        nshot2 = nshot1 + nshots // nprocshot + 1
    else:
        nshot1 += nshots % nprocshot
        nshot2 = nshot1 + nshots // nprocshot
    return nshot1 + 1, nshot2 + 1


@pytest.mark.parametrize("world,nprocfreq", [(1, 1), (4, 2), (6, 3), (6, 1), (8, 8), (8, 2)])
@pytest.mark.parametrize("nf,nshots", [(10, 100), (3, 7), (1, 5)])
def test_rank_blocks_is_reference_layout(world, nprocfreq, nf, nshots):
    """COLOR = MYID / NPROCFREQ, MYID_SHOT = MYID % NPROCFREQ
    (src/AC/fwi_FD_AC.c:201-211); every (frequency, shot) pair on exactly
    one rank."""
    seen = np.zeros((nf, nshots), int)
    for myid in range(world):
        (flo, fhi), (slo, shi) = rank_blocks(nf, nshots, world, myid, nprocfreq)
        color, myid_shot = myid // nprocfreq, myid % nprocfreq
        n1, n2 = init_mpifreq(nf, nprocfreq, myid_shot)
        s1, s2 = init_mpishot(nshots, world // nprocfreq, color)
        assert (flo, fhi, slo, shi) == (n1 - 1, n2 - 1, s1 - 1, s2 - 1)
        seen[flo:fhi, slo:shi] += 1
    assert np.all(seen == 1)


def test_rank_blocks_rejects_uneven_layout():
    with pytest.raises(ValueError):
        rank_blocks(10, 100, 6, 0, 4)
    with pytest.raises(ValueError):
        rank_blocks(10, 100, 4, 4, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    from tests.models import inclusion_ac, random_smooth
    import oracle as O
    nx, ny, dh, npml = 40, 30, 10.0, 6
    vp, rho = inclusion_ac(nx, ny, dh, npml, radius=50.0)
    vp = vp * random_smooth(nx, ny, 0.9, 1.1, 4)
    g = O.Grid(nx=nx, ny=ny, dh=dh, npml=npml)
    nx0 = nx - 2 * npml
    xs = np.linspace(2 * dh, (nx0 - 3) * dh, 3).astype(np.float32)
    ys = np.full(3, 3 * dh, np.float32)
    rx = np.arange(1, nx0 - 1, dtype=np.int32)
    ry = np.full(rx.size, 3, np.int32)
    freqs = [6.0, 9.0, 13.0]
    return g, vp, rho, xs, ys, rx, ry, freqs


def _oracle_local(g, vp, rho, xs, ys, rx, ry, obs_by_freq):
    from tests.test_gpu_forward_grad import oracle_grad

    def run(local, shots=None):
        sel = slice(None) if shots is None else slice(shots.start, shots.stop)
        if not local or (shots is not None and len(shots) == 0):
            return np.zeros(g.n), None, 0.0
        obs = np.stack([obs_by_freq[f][sel] for f in local])
        g0, _, l2 = oracle_grad(g, 1, vp, rho, local, xs[sel], ys[sel], rx, ry, obs, 0, 1)
        return g0, None, l2
    return run


def _observed(g, vp, rho, xs, ys, rx, ry, freqs):
    from tests.test_gpu_forward_grad import _observed as obs_fn
    obs = obs_fn(g, 1, vp, rho, freqs, xs, ys, rx, ry)
    return {f: obs[i] for i, f in enumerate(freqs)}


def _worker(rank, world, port, out_dir, npf=None):
    import torch.distributed as dist
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        g, vp, rho, xs, ys, rx, ry, freqs = _case()
        obs = _observed(g, vp, rho, xs, ys, rx, ry, freqs)
        g0, _, l2 = sharded_grad_obj(freqs, _oracle_local(g, vp, rho, xs, ys, rx, ry, obs), dist,
                                     nshots=xs.size, nprocfreq=npf)
        np.save(os.path.join(out_dir, f"g{rank}.npy"), np.append(g0, l2))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,npf", [(2, None), (4, None), (4, 2), (6, 2)],
                         ids=["w2", "w4-idle-rank", "w4-2x2-shots", "w6-2x3-shots"])
def test_sharded_gradient_gloo_equals_single_process(world, npf):
    """world 2: shares of 2 and 1 frequencies; world 4: one rank has none;
    2 x 2 and 2 x 3: two frequency blocks with their 3 shots split over 2 or
    3 ranks (the reference's NPROCSHOT)."""
    import torch.multiprocessing as tmp
    with tempfile.TemporaryDirectory() as d:
        tmp.spawn(_worker, args=(world, _free_port(), d, npf), nprocs=world, join=True)
        res = [np.load(os.path.join(d, f"g{r}.npy")) for r in range(world)]
    g, vp, rho, xs, ys, rx, ry, freqs = _case()
    obs = _observed(g, vp, rho, xs, ys, rx, ry, freqs)
    g_all, _, l2_all = _oracle_local(g, vp, rho, xs, ys, rx, ry, obs)(freqs)
    for r in res:   # every rank holds the same total
        assert np.array_equal(r, res[0])
    assert np.linalg.norm(res[0][:-1] - g_all) <= 1e-12 * np.linalg.norm(g_all)
    assert abs(res[0][-1] - l2_all) <= 1e-12 * abs(l2_all)


def test_local_frequencies_slices():
    f = [2.0, 3.0, 4.0, 5.0, 6.0]
    assert local_frequencies(f, 2, 0) == [2.0, 3.0, 4.0]
    assert local_frequencies(f, 2, 1) == [5.0, 6.0]
    assert local_frequencies(f, 8, 7) == []


@pytest.mark.gpu
def test_sharded_engine_gradient_over_nccl():
    """One rank over NCCL on cuda:0: the all-reduce of the engine's FP64
    gradient (device buffer) returns it unchanged and equals the oracle; the
    engine's share over two shot blocks (what two ranks of one frequency
    block evaluate) sums to the whole."""
    import datetime
    import torch
    import torch.distributed as dist
    from germaine_b200 import Engine
    from germaine_b200.sharding import engine_grad_obj
    g, vp, rho, xs, ys, rx, ry, freqs = _case()
    obs = _observed(g, vp, rho, xs, ys, rx, ry, freqs)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        with Engine(g.nx, g.ny, g.dh, g.npml, leaf_max=32) as e:
            e.set_model(vp, rho)
            run = engine_grad_obj(e, xs, ys, rx, ry, obs)
            g0, _, l2 = sharded_grad_obj(freqs, run, dist, device=torch.device("cuda", 0))
            ga, _, la = run(freqs, range(0, 2))
            gb, _, lb = run(freqs, range(2, 3))
    finally:
        dist.destroy_process_group()
    assert np.linalg.norm(ga + gb - g0) <= 1e-10 * np.linalg.norm(g0)
    assert abs(la + lb - l2) <= 1e-5 * abs(l2)
    r0, _, rl2 = _oracle_local(g, vp, rho, xs, ys, rx, ry, obs)(freqs)
    assert np.linalg.norm(g0 - r0) <= 1e-8 * np.linalg.norm(r0)
    assert abs(l2 - rl2) <= 2e-6 * abs(rl2)


def _seis_block(f, nshots, ntr):
    """Seeded seismograms of frequency index f, with a few signed zeros."""
    rng = np.random.default_rng(100 + f)
    s = (rng.standard_normal((nshots, ntr)) + 1j * rng.standard_normal((nshots, ntr))).astype(np.complex64)
    s[0, 0] = np.complex64(complex(-0.0, -0.0))
    s[-1, -1] = np.complex64(complex(0.0, -0.0))
    return s


def _gather_worker(rank, world, port, out_dir, nf, nshots, ntr, npf):
    import torch.distributed as dist
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        (lo, hi), (slo, shi) = rank_blocks(nf, nshots, world, rank, npf)
        loc = np.stack([_seis_block(f, nshots, ntr)[slo:shi] for f in range(lo, hi)]) if hi > lo else None
        out = gather_seismograms(loc, nf, nshots, ntr, dist, nprocfreq=npf)
        np.save(os.path.join(out_dir, f"s{rank}.npy"), out)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nf,nshots,npf", [(2, 3, 3, None), (3, 4, 3, None), (4, 3, 3, None), (4, 3, 5, 2),
                                                 (6, 2, 7, 3)],
                         ids=["w2-nf3", "w3-nf4", "w4-nf3-idle-rank", "w4-2x2-shots", "w6-3x2-idle-freq"])
def test_gather_seismograms_gloo_equals_reference_sum(world, nf, nshots, npf):
    """Uneven shares, ranks without frequencies, and split shots
    (NPROCFREQ = npf); every rank ends with what summing zero-filled full
    arrays over the ranks gives, bit for bit (signed zeros included)."""
    import torch.multiprocessing as tmp
    ntr = 5
    with tempfile.TemporaryDirectory() as d:
        tmp.spawn(_gather_worker, args=(world, _free_port(), d, nf, nshots, ntr, npf), nprocs=world, join=True)
        res = [np.load(os.path.join(d, f"s{r}.npy")) for r in range(world)]
    ref = np.zeros((nf, nshots, ntr), np.complex64)   # write_seis_AC: sum of each rank's zero-filled array
    for r in range(world):
        (lo, hi), (slo, shi) = rank_blocks(nf, nshots, world, r, npf)
        part = np.zeros_like(ref)
        for f in range(lo, hi):
            part[f, slo:shi] = _seis_block(f, nshots, ntr)[slo:shi]
        ref = ref + part
    for out in res:
        assert out.shape == (nf, nshots, ntr)
        assert out.view(np.uint32).tobytes() == ref.view(np.uint32).tobytes()


def _oracle_forward_local(g, vp, rho, xs, ys, rx, ry):
    from tests.test_gpu_forward_grad import oracle_forward
    from oracle import sparse as OS
    idx = [OS.receiver_read_index(g, int(a), int(b)) for a, b in zip(rx, ry)]

    def run(local, shots=None):
        sel = slice(None) if shots is None else slice(shots.start, shots.stop)
        if not local or (shots is not None and len(shots) == 0):
            return None
        X, _ = oracle_forward(g, 1, vp, rho, local, xs[sel], ys[sel])
        return np.stack([OS.vec2mat(X[i].T)[:, idx] for i in range(len(local))]).astype(np.complex64)
    return run


def _forward_worker(rank, world, port, out_dir, npf):
    import torch.distributed as dist
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        g, vp, rho, xs, ys, rx, ry, freqs = _case()
        seis = sharded_forward(freqs, _oracle_forward_local(g, vp, rho, xs, ys, rx, ry), xs.size, rx.size, dist,
                               nprocfreq=npf)
        np.save(os.path.join(out_dir, f"f{rank}.npy"), seis)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,npf", [(2, None), (4, None), (4, 2)], ids=["w2", "w4-idle-rank", "w4-2x2-shots"])
def test_sharded_forward_gloo_equals_single_process(world, npf):
    """world 2: shares of 2 and 1 frequencies; world 4: one rank has none;
    2 x 2: two frequency blocks, each with its shots split over two ranks
    (their solves take fewer right-hand sides at once, so equal to the
    float32 rounding of the seismograms)."""
    import torch.multiprocessing as tmp
    with tempfile.TemporaryDirectory() as d:
        tmp.spawn(_forward_worker, args=(world, _free_port(), d, npf), nprocs=world, join=True)
        res = [np.load(os.path.join(d, f"f{r}.npy")) for r in range(world)]
    g, vp, rho, xs, ys, rx, ry, freqs = _case()
    ref = _oracle_forward_local(g, vp, rho, xs, ys, rx, ry)(freqs) + np.complex64(0)
    for out in res:
        assert out.tobytes() == res[0].tobytes()
        if npf is None:
            assert np.array_equal(out, ref)
        else:
            assert np.linalg.norm(out - ref) <= 1e-6 * np.linalg.norm(ref)


@pytest.mark.gpu
def test_sharded_engine_forward_over_nccl():
    """One rank over NCCL on cuda:0: the gathered seismograms (device
    buffers) are the engine's own block, bit for bit, and match the oracle;
    the engine's share for a shot block is that block of the whole."""
    import datetime
    import torch
    import torch.distributed as dist
    from germaine_b200 import Engine
    from germaine_b200.sharding import engine_forward
    g, vp, rho, xs, ys, rx, ry, freqs = _case()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        with Engine(g.nx, g.ny, g.dh, g.npml, leaf_max=32) as e:
            e.set_model(vp, rho)
            run, blocks = engine_forward(e, xs, ys, rx, ry), []

            def local(fs, shots):
                blocks.append(run(fs, shots))
                return blocks[-1]
            seis = sharded_forward(freqs, local, xs.size, rx.size, dist, device=torch.device("cuda", 0))
            part = run(freqs, range(1, 3))
    finally:
        dist.destroy_process_group()
    assert np.array_equal(seis, blocks[0])
    assert np.linalg.norm(part - seis[:, 1:3]) <= 1e-6 * np.linalg.norm(seis[:, 1:3])
    ref = _oracle_forward_local(g, vp, rho, xs, ys, rx, ry)(freqs)
    assert np.linalg.norm(seis - ref) <= 2e-6 * np.linalg.norm(ref)


def _failure_worker(rank, world, port, out_dir, mode):
    """Rank 1 fails its local step (mode "raise"), returns seismograms of
    the wrong shape (mode "shape"), or stalls past the process group's
    timeout before it (mode "stall"); every rank records what it raised and
    when."""
    import time
    import torch.distributed as dist
    import datetime
    from germaine_b200.sharding import RankFailure
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=3))
    freqs = [2.0, 3.0, 4.0]

    def local(fs, shots):
        if rank == 1 and mode == "raise":
            raise FloatingPointError("singular front")
        if rank == 1 and mode == "stall":
            time.sleep(8)
        return np.zeros(16), None, float(len(fs))
    def local_seis(fs, shots):   # rank 1 returns a block of the wrong shape
        return np.zeros((len(fs), 4 if rank == 1 else 3, 5), np.complex64)
    t0 = time.monotonic()
    try:
        if mode == "shape":
            sharded_forward(freqs, local_seis, 3, 5, dist)
        else:
            sharded_grad_obj(freqs, local, dist)
        what = "ok"
    except RankFailure:
        what = "RankFailure"
    except (FloatingPointError, ValueError):
        what = "own"
    except RuntimeError:   # the process group's timeout or a closed peer
        what = "timeout"
    took = time.monotonic() - t0
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(f"{what} {took:.2f}")
    if mode != "stall":
        dist.destroy_process_group()


def _outcomes(world, mode):
    import torch.multiprocessing as tmp
    with tempfile.TemporaryDirectory() as d:
        tmp.spawn(_failure_worker, args=(world, _free_port(), d, mode), nprocs=world, join=True)
        out = []
        for r in range(world):
            what, took = open(os.path.join(d, f"r{r}.txt")).read().split()
            out.append((what, float(took)))
    return out


@pytest.mark.parametrize("mode", ["raise", "shape"])
def test_sharded_rank_failure_reaches_every_rank(mode):
    """A rank whose evaluation raises (or returns seismograms of the wrong
    shape) still takes the failure-count step: it re-raises its own error,
    every other rank raises RankFailure at the same step, and none waits
    for the timeout."""
    out = _outcomes(3, mode)
    assert [w for w, _ in out] == ["RankFailure", "own", "RankFailure"]
    assert all(t < 2.5 for _, t in out), out


def test_sharded_stalled_rank_ends_in_the_timeout():
    """A rank that stalls past the process group's timeout: the waiting
    rank's collective ends with an error instead of hanging."""
    out = _outcomes(2, "stall")
    assert out[0][0] == "timeout" and out[0][1] < 7.5, out
