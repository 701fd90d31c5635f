"""Benchmark: shot-solves/s of the per-frequency factor + solve path on B200.

Workload (default): the 801 x 187 synthetic thrust model at DH = 25 m with a
20-point PML (841 x 227 grid, N = 190,907 unknowns), 10 frequencies
2, 3, ..., 11 Hz, 100 shots along model row 2, 800 receivers on the same row.
One step = assemble + factorise all 10 frequencies + solve all 100 shots of
every frequency (1,000 shot-solves) with FP64 iterative refinement to a
relative residual <= 1e-10, and gather the seismograms.

Both paths are run on the same step:
  fp64   -- the drop-in: complex128 fronts and substitution, one FP64
            residual check (refinement only if it is above the target);
  mixed  -- complex64 fronts and substitution with FP64 iterative
            refinement (residual and update in FP64) to the same target.

  value  -- the faster of the two (config.path names it), inputs and outputs
            resident in HBM, device time from CUDA events on the engine's
            stream; `paths` reports both, `mixed_over_fp64` their ratio;
  e2e    -- the same path and step through the public C-ABI with host
            buffers: the model is copied in from pinned host memory and the
            seismograms copied back every step, inside the timed region.

`--impl reference` times the reference's CPU path on the host cores: the
reference's own assembly (oracle/_ref, else the C restatement) and SciPy
SuperLU standing in for UMFPACK, one process per frequency with all of its
shots (the reference's MPI frequency/shot split on one node).

Multi-GPU: each rank runs the full step on its own GPU (independent
frequency batches, no data-path collective: weak scaling); the step time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DH, NPML, ROW = 25.0, 20, 2
RESIDUAL_TARGET = 1e-10
METRIC = "shot-solves/s (factor+solve) mixed vs FP64 on B200 at resid<=1e-10; %roofline"
# DRAM bytes of one complex128 backward substitution pass on 4 frequencies
# (the k_bwd_small / k_bwd_ring / k_bwd_piv launches of the FP64 engine's
# timed step, ncu dram__bytes_read.sum + dram__bytes_write.sum, summed)
BWD_TRAFFIC_FP64_4FREQ = 3.585e9
PEAK_KIND = "measured FP64 rate, the higher of CUDA-core DFMA (gm_peak_fp64) and FP64 MMA (gm_peak_fp64_mma)"

# the benchmark workload; --nx0/--ny0/--nfreq/--nshots shrink it for
# profiling captures (the bench line then names the smaller workload)
W = {"nx0": 801, "ny0": 187, "nfreq": 10, "nshots": 100}


def freqs_hz() -> list[float]:
    return [float(f) for f in range(2, 2 + W["nfreq"])]


def workload_name() -> str:
    nx, ny = W["nx0"] + 2 * NPML, W["ny0"] + 2 * NPML
    f = freqs_hz()
    return (f"thrust {W['nx0']}x{W['ny0']} h=25m pml20 ({nx}x{ny}, N={nx * ny}), "
            f"{len(f)} freqs {f[0]:g}-{f[-1]:g} Hz x {W['nshots']} shots, {W['nx0'] - 1} receivers, AC")


def workload(seed: int = 2024):
    from germaine_b200.synthetic import line_acquisition, thrust_model
    vp, rho = thrust_model(W["nx0"], W["ny0"], DH, NPML, seed=seed)
    xs, ys, rx, ry = line_acquisition(W["nx0"], DH, W["nshots"], ROW)
    return vp, rho, xs, ys, rx, ry


# ----------------------------------------------------------------- CPU arm
def _cpu_rank(args):
    """One MPI rank of the CPU reference path: for each of its frequencies,
    assemble (the reference's own sources), factorise M = A^T with SuperLU
    and solve its shots.  Returns (wall seconds, factor seconds, solve
    seconds, shot-solves done)."""
    freqs, shots, seed, dims = args
    W.update(dims)
    import oracle as O
    from oracle import sparse as OS
    vp, rho, xs, ys, rx, ry = workload(seed)
    g = O.Grid(nx=W["nx0"] + 2 * NPML, ny=W["ny0"] + 2 * NPML, dh=DH, npml=NPML)
    asm = O.Ref(g) if O.ref_available() else O.Port(g)
    idx = [OS.receiver_read_index(g, int(a), int(b)) for a, b in zip(rx, ry)]
    t0 = time.perf_counter()
    tf = ts = 0.0
    for freq in freqs:
        a = time.perf_counter()
        trip = asm.assemble(1, freq, vp, rho)
        ds = OS.DirectSolver(OS.operator(OS.assembled_matrix(g, *trip)))
        b = time.perf_counter()
        if shots:
            B = OS.spike_rhs(g, 1, freq, xs[shots], ys[shots])
            X = ds.solve(B)
            _ = OS.vec2mat(X.T)[:, idx]
        ts += time.perf_counter() - b
        tf += b - a
    return time.perf_counter() - t0, tf, ts, len(freqs) * len(shots)


def rank_work(nprocfreq: int, nprocshot: int, nshots: int):
    """Per-rank (frequencies, shots) of the reference's layout: rank MYID in
    colour MYID / NPROCFREQ takes the shot block of its colour and the
    frequency block of its rank in the colour (fwi_FD_AC.c:201-211,
    init_MPIfreq.c:20-31, init_MPIshot.c:20-31)."""
    from germaine_b200.sharding import rank_blocks
    fl = freqs_hz()
    world = nprocfreq * nprocshot
    work = []
    for myid in range(world):
        (flo, fhi), (slo, shi) = rank_blocks(len(fl), nshots, world, myid, nprocfreq)
        work.append((fl[flo:fhi], list(range(slo, shi))))
    return work


def choose_layout(cores: int, nshots: int, t_factor: float, t_shot: float):
    """The reference layout (NPROCFREQ x NPROCSHOT ranks <= cores) with the
    least per-rank time under the measured factor / per-shot costs."""
    best = None
    for pf in range(1, cores + 1):
        for ps in range(1, cores // pf + 1):
            cost = max(len(fr) * (t_factor + len(sh) * t_shot) for fr, sh in rank_work(pf, ps, nshots) if fr or sh)
            key = (cost, pf * ps)
            if best is None or key < best[0]:
                best = (key, pf, ps)
    return best[1], best[2]


def _one_blas_thread():
    saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
    for k in saved:
        os.environ[k] = "1"
    return saved


def _restore(saved):
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


def cpu_probe(seed: int = 2024, nshots: int = 10):
    """Factor and per-shot solve cost of one frequency in one process."""
    saved = _one_blas_thread()
    try:
        with mp.get_context("spawn").Pool(1) as pool:
            _, tf, ts, done = pool.map(_cpu_rank, [([freqs_hz()[len(freqs_hz()) // 2]],
                                                    list(range(min(nshots, W["nshots"]))), seed, dict(W))])[0]
    finally:
        _restore(saved)
    return tf, ts / max(1, done)


def cpu_reference_step(layout, nshots: int | None = None, seed: int = 2024):
    """One bounded sample: the reference's MPI layout (NPROCFREQ,
    NPROCSHOT) as processes, one BLAS thread each.  Returns (shot-solves/s,
    wall seconds, shot-solves done)."""
    nshots = nshots or W["nshots"]
    pf, ps = layout
    jobs = [(fr, sh, seed, dict(W)) for fr, sh in rank_work(pf, ps, nshots) if fr]
    saved = _one_blas_thread()
    try:
        t0 = time.perf_counter()
        with mp.get_context("spawn").Pool(len(jobs)) as pool:
            res = pool.map(_cpu_rank, jobs)
        wall = time.perf_counter() - t0
    finally:
        _restore(saved)
    done = sum(r[3] for r in res)
    return done / wall, wall, done


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline_kind() -> str:
    import oracle as O
    return "reference" if O.ref_available() else "port"


def cpu_setup():
    """Cores, the chosen reference layout and its description."""
    cores = os.cpu_count() or 1
    tf, tshot = cpu_probe()
    pf, ps = choose_layout(cores, W["nshots"], tf, tshot)
    desc = (f"reference MPI layout NPROCFREQ={pf} x NPROCSHOT={ps} on {cores} host cores ({cpu_model()}); "
            f"assembly from the reference's own sources, SciPy SuperLU standing in for UMFPACK (absent on the "
            f"GPU host); probe: factor {tf:.2f} s, {1e3 * tshot:.1f} ms per shot")
    return (pf, ps), pf * ps, desc


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------- GPU arm
def time_steps(torch, e, step, steps: int, warmup: int, dist=None, tag: str = "timed"):
    """Device time per step over `steps` steps after `warmup` untimed ones;
    the timed steps sit in an NVTX range named `tag` (profilers can select
    them, e.g. ncu --nvtx --nvtx-include "timed_fp64/")."""
    for _ in range(warmup):
        step()
    stream = torch.cuda.ExternalStream(e.stream())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    l0 = e.stats()["kernel_launches"]
    torch.cuda.nvtx.range_push(tag)
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    if dist is not None:
        dist.barrier()
    ms = ev0.elapsed_time(ev1) / steps
    launches = (e.stats()["kernel_launches"] - l0) // steps
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, int(launches)


def measure_fp64_peak(device: int):
    """FP64 rates (TFLOP/s) measured by the library's microbenchmarks before
    any timed step: (CUDA-core DFMA, FP64 matrix instructions)."""
    import ctypes

    from germaine_b200 import _lib
    lib = _lib.load()
    fma, mma = ctypes.c_double(0.0), ctypes.c_double(0.0)
    _lib.check(lib.gm_peak_fp64(device, ctypes.byref(fma)))
    _lib.check(lib.gm_peak_fp64_mma(device, ctypes.byref(mma)))
    return float(fma.value), float(mma.value)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, "fallback"


def run_gpu(args):
    import torch

    from germaine_b200 import GM_PREC_C64_IR, GM_PREC_FP64, Engine
    from germaine_b200._lib import GM_WARNING_NOT_CONVERGED

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod
        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod
    else:
        torch.cuda.set_device(local)

    # CPU baseline first (spawned processes before heavy GPU work)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        layout, ncores, desc = cpu_setup()
        rate, wall, done = cpu_reference_step(layout)
        cpu = {"value": rate, "unit": "shot-solves/s", "cores": ncores, "kind": cpu_baseline_kind(),
               "sample": f"the whole workload ({done} shot-solves, {W['nfreq']} frequencies); {desc}; "
                         f"wall {wall:.1f} s"}

    vp, rho, xs, ys, rx, ry = workload(args.seed + rank)
    nx, ny = W["nx0"] + 2 * NPML, W["ny0"] + 2 * NPML
    freqs = np.array(freqs_hz(), np.float32)
    nf, ns, ntr = len(freqs), W["nshots"], rx.size
    dev = torch.device("cuda", local)
    vp_d = torch.from_numpy(vp.reshape(-1)).to(dev)
    rho_d = torch.from_numpy(rho.reshape(-1)).to(dev)
    seis_d = torch.empty((nf, ns, ntr, 2), dtype=torch.float32, device=dev)
    vp_h = torch.from_numpy(vp.reshape(-1)).pin_memory()
    rho_h = torch.from_numpy(rho.reshape(-1)).pin_memory()
    seis_h = torch.empty((nf, ns, ntr, 2), dtype=torch.float32).pin_memory()
    peak_hbm, peak_bf16, peak_kind = load_peaks()
    fp64_fma_peak, fp64_mma_peak = measure_fp64_peak(local)
    # the complex128 kernels run on both instruction kinds: the higher
    # measured rate is the denominator (the lower fraction)
    fp64_peak = max(fp64_fma_peak, fp64_mma_peak)

    results = {}
    for name, prec in (("mixed", GM_PREC_C64_IR), ("fp64", GM_PREC_FP64)):
        e = Engine(nx, ny, DH, NPML, precision=prec, device=local, leaf_max=args.leaf,
                   refine={"auto": 0, "ir": 1, "gmres": 2}[args.refine])
        e.set_model(vp_d, rho_d)
        tuned = None
        if args.autotune:   # substitution tiles per level, timed on this workload's factors (untimed set-up)
            e.factor(freqs)
            tuned = e.autotune(ns)

        def check_converged(tag):
            # every step must meet the residual target: a path that stops
            # above it (GM_WARNING_NOT_CONVERGED) has no valid number
            st = e.stats()
            if e.last_status == GM_WARNING_NOT_CONVERGED or not st["ir_residual"] <= RESIDUAL_TARGET:
                raise SystemExit(f"bench: {name} path ({tag}) did not reach the residual target: status "
                                 f"{e.last_status}, max relative residual {st['ir_residual']:.3e}")

        def step_dev():
            e.factor(freqs)
            e.forward(xs, ys, rx, ry, seis_out=seis_d)
            check_converged("device-resident")

        clocks = ClockSampler(local)
        clocks.start()
        ms, launches = time_steps(torch, e, step_dev, args.steps, args.warmup, dist, tag=f"timed_{name}")
        ck = clocks.stop()
        st = e.stats()
        r = {"ms": ms, "launches": launches, "stats": st, "clocks": ck, "tuned": tuned}

        def step_e2e():
            e.set_model(vp_h, rho_h)
            e.factor(freqs)
            e.forward(xs, ys, rx, ry, seis_out=seis_h)
            check_converged("end-to-end")
        ms_e2e, _ = time_steps(torch, e, step_e2e, max(1, args.steps // 2), 1, dist, tag=f"e2e_{name}")
        r["ms_e2e"] = ms_e2e
        # per-frequency refinement record of the last step and, outside the
        # timed region, the FP64 forward wavefields for the error table
        r["refine"] = e.refine_report()
        r["x"] = e.wavefield_fp64(0, ns) if args.wavefield_error else None
        results[name] = r
        e.close()
        del e
        torch.cuda.empty_cache()

    mixed, fp64 = results["mixed"], results["fp64"]
    per_freq = []
    for i, f in enumerate(freqs):
        row = {"freq_hz": float(f)}
        for nm in ("mixed", "fp64"):
            rf = results[nm]["refine"][i]
            row[nm] = {"first_residual": rf["first_residual"], "final_residual": rf["final_residual"],
                       "sweeps": rf["sweeps"], "method": rf["method"]}
        if mixed["x"] is not None:
            a, b = mixed["x"][i], fp64["x"][i]
            row["mixed_wavefield_rel_l2_vs_fp64"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
        per_freq.append(row)
    for nm in ("mixed", "fp64"):
        results[nm]["x"] = None
    units = nf * ns * world
    # headline: the faster of the two paths (both refine to the residual
    # target); the other is reported beside it
    head_name = "fp64" if fp64["ms"] <= mixed["ms"] else "mixed"
    head = results[head_name]
    value = units / (head["ms"] * 1e-3)
    st = head["stats"]
    # roofline of the backward substitution pass (K5 k_bwd_small on the
    # fronts with at most 32 pivots, k_bwd_ring + k_bwd_piv above them;
    # the dense part of every solve: the forward pass is pruned to the
    # fronts on the paths from the sources to the root): the stored U
    # entries read once + the right-hand sides read (y, ancestors' x) and the
    # solution written, over the device time of the backward passes
    csize = 16 if head_name == "fp64" else 8
    subst_bytes = nf * (st["u_entries"] * csize + 2 * st["n"] * ns * csize)
    subst_ms = st["ms_subst_bwd"] / max(1, st["n_subst"])
    achieved = subst_bytes / (subst_ms * 1e-3) / 1e9
    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one
    # backward pass from an ncu capture of this workload on 4 frequencies,
    # scaled by frequency count
    per4 = {"mixed": None, "fp64": BWD_TRAFFIC_FP64_4FREQ}[head_name]
    traffic = (per4 / 4 * nf if per4 and (W["nx0"], W["ny0"], W["nshots"], args.leaf) == (801, 187, 100, 32)
               else None)
    # the same pass against the FP64 (complex64: FP32) CUDA-core rate -- at
    # 100 right-hand sides its arithmetic intensity (8 flops per stored U
    # entry per right-hand side) is above the HBM ridge -- and the
    # factorisation against it: exact flop counts of the symbolic analysis
    # over the device time of the phase
    subst_flops = 8.0 * st["u_entries"] * ns * nf
    factor_flops = st["factor_flops"] * nf
    peak_fp = fp64_peak * (2.0 if head_name == "mixed" else 1.0)
    roofline_compute = [
        {"kernel": "K5 backward substitution (same launch group)", "bound": "fp64" if csize == 16 else "fp32",
         "achieved": subst_flops / (subst_ms * 1e-3) / 1e12, "peak": peak_fp, "unit": "TFLOP/s",
         "frac": subst_flops / (subst_ms * 1e-3) / 1e12 / peak_fp, "algorithmic_flops": subst_flops,
         "arithmetic_intensity_flop_per_byte": subst_flops / subst_bytes,
         "peak_kind": PEAK_KIND + (" x 2 for FP32" if csize == 8 else "")},
        {"kernel": "K2-K4 factorisation, all levels", "bound": "fp64" if csize == 16 else "fp32",
         "achieved": factor_flops / (st["ms_factor"] * 1e-3) / 1e12, "peak": peak_fp, "unit": "TFLOP/s",
         "frac": factor_flops / (st["ms_factor"] * 1e-3) / 1e12 / peak_fp, "algorithmic_flops": factor_flops,
         "ms": st["ms_factor"], "peak_kind": PEAK_KIND + (" x 2 for FP32" if csize == 8 else "")},
    ]
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "shot-solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": head["ms"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c128" if head_name == "fp64" else "c64 fronts + f64 refinement",
        "data": "synthetic (seeded thrust model; no public dataset)",
        "config": {"workload": workload_name(), "frequencies": nf, "shots_per_frequency": ns, "receivers": ntr,
                   "path": {"fp64": "FP64 drop-in (complex128 factors and substitution, FP64 residual check)",
                            "mixed": "complex64 factors + FP64 iterative refinement"}[head_name],
                   "residual_target": 1e-10, "l2": "inputs larger than L2 (fronts 4-8 GB per step)",
                   "parallelism": f"replicas{world}" if world > 1 else "single"},
        "e2e": {"value": units / (head["ms_e2e"] * 1e-3), "unit": "shot-solves/s",
                "h2d_bytes_per_step": int(2 * vp.size * 4), "d2h_bytes_per_step": int(nf * ns * ntr * 8)},
        "paths": {n: {"value": units / (results[n]["ms"] * 1e-3), "ms_per_step": results[n]["ms"],
                      "e2e_value": units / (results[n]["ms_e2e"] * 1e-3),
                      "ir_iterations": results[n]["stats"]["ir_iterations"],
                      "ir_residual": results[n]["stats"]["ir_residual"],
                      "perturbed_pivots": results[n]["stats"]["perturbed_pivots"],
                      "phase_ms": {"assemble": results[n]["stats"]["ms_assemble"],
                                   "factor": results[n]["stats"]["ms_factor"],
                                   "solve": results[n]["stats"]["ms_solve"],
                                   "refine": results[n]["stats"]["ms_refine"],
                                   "substitutions": results[n]["stats"]["ms_subst"],
                                   "n_subst": results[n]["stats"]["n_subst"]},
                      "gpu_launches_per_step": results[n]["launches"],
                      "autotuned_tiles": results[n]["tuned"]}
                  for n in ("fp64", "mixed")},
        "mixed_over_fp64": fp64["ms"] / mixed["ms"],
        "per_frequency": per_freq,
        "roofline": {"kernel": "K5 backward substitution (k_bwd_small, k_bwd_ring + k_bwd_piv, %s)" % ("complex128" if csize == 16 else "complex64"),
                     "bound": "hbm", "achieved": achieved, "peak": peak_hbm, "unit": "GB/s",
                     "frac": achieved / peak_hbm, "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes": subst_bytes, "ms_per_launch_group": subst_ms},
        "roofline_compute": roofline_compute,
        "fp64_peak_tflops": {"dfma": fp64_fma_peak, "mma": fp64_mma_peak},
        "gpu_launches": head["launches"] * args.steps,
        "clocks": head["clocks"],
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    layout, ncores, desc = cpu_setup()
    for _ in range(args.warmup):
        cpu_reference_step(layout, nshots=min(W["nshots"], 10))
    rates, walls = [], []
    # each step is the whole workload (about 6-10 s on a 16-core host)
    for _ in range(args.steps):
        r, w, _ = cpu_reference_step(layout)
        rates.append(r)
        walls.append(w)
    value = float(np.median(rates))
    line = {
        "metric": METRIC, "value": value, "unit": "shot-solves/s", "n_gpus": int(os.environ.get("WORLD_SIZE", 1)),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.median(walls)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded thrust model; no public dataset)",
        "config": {"workload": workload_name(), "frequencies": W["nfreq"], "shots_per_frequency": W["nshots"]},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "shot-solves/s", "cores": ncores, "kind": cpu_baseline_kind(),
                         "sample": f"{len(rates)} step(s) of the whole workload; {desc}"},
        "e2e": {"value": value, "unit": "shot-solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--leaf", type=int, default=32)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--refine", choices=["auto", "ir", "gmres"], default="auto",
                    help="refinement of the mixed path: automatic IR / GMRES-IR choice, IR only, GMRES-IR only")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default substitution tiles instead of the per-level autotuned ones")
    ap.add_argument("--no-wavefield-error", dest="wavefield_error", action="store_false",
                    help="skip the per-frequency wavefield comparison of the two paths (outside the timed region)")
    ap.add_argument("--nx0", type=int, default=W["nx0"], help="model width without PML (profiling cases)")
    ap.add_argument("--ny0", type=int, default=W["ny0"], help="model depth without PML (profiling cases)")
    ap.add_argument("--nfreq", type=int, default=W["nfreq"], help="frequencies 2, 3, ... Hz (profiling cases)")
    ap.add_argument("--nshots", type=int, default=W["nshots"], help="shots per frequency (profiling cases)")
    args = ap.parse_args()
    W.update(nx0=args.nx0, ny0=args.ny0, nfreq=args.nfreq, nshots=args.nshots)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
