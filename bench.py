"""Throughput of the FELIS slice loop on B200.

Workload (default `sase`): time-dependent SASE, 8 GeV beam, flat-top 3 kA
over 1024 slices of 8192 particles (8,388,608 in all) with shot-noise
phases, BiPolar undulator lambda_u = 2.6 cm, K0 = 2.6, 102 x 102 grid over
+-300 um, one step per undulator period.  A "step" is one iteration of the
reference loop (main.cpp:117-155) over every slice.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl felis|reference]

--impl felis      the GPU library.  The headline `value` is the
                  mixed-precision engine (felis_batch_*: FP32 push and ADI,
                  FP64 theta and reductions) on the workload; beside it, the
                  FP64 plain path on the same workload (`fp64_plain`), the
                  speed-up and the power error between the two, and the
                  96-instance batched ensemble (`ensemble`).  Each path runs W
                  untimed iterations, then K iterations replayed from one CUDA
                  graph, timed with CUDA events on the library's stream
                  (inputs resident in HBM); `e2e` is the mixed engine end to
                  end through the C ABI with host buffers; the CPU
                  restatement runs on a bounded sample as a reported baseline.
--impl reference  the reference's CPU path (the oracle port: the reference
                  does not build here, it needs MPI/HDF5/GSL) on the host's
                  cores, on a bounded sample of the same workload.
Under torchrun (N > 1) every rank runs its own copy of the workload on its
GPU (weak scaling); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s + ADI cells/s vs FP64 plain GPU path at <=1% power error"
UNIT = "particle-steps/s"
BYTES_PARTICLE_STEP = 96   # FP64: read + write 6 x 8 B of state
BYTES_ADI_CELL = 32        # FP64: read + write one complex cell


def peaks() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def tensor_peak() -> tuple[float, str]:
    """Dense BF16 TFLOP/s: the measured burst figure, else the fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def run_surrogate_gemm(rows: int, chain_too: bool = True, fused: bool = True) -> dict:
    """The taper surrogate ranking `rows` candidate tapers: the inference pass
    38 -> 256 -> 256 -> 256 -> 33 (BF16 operands, FP32 accumulation on the
    tensor cores) as one fused kernel (activations on chip) and, for
    comparison, as the layer-by-layer GEMM chain; each timed with CUDA events
    on the network's stream, best of three after one untimed pass."""
    import numpy as np

    import felis_b200 as fb

    m = fb.MLP(38, 256, 33, seed=3)
    x = np.random.default_rng(1).standard_normal((rows, 38)).astype(np.float32)

    def timed(use_fused):
        m.set_fused(use_fused)
        m.forward(x)
        best = None
        for _ in range(3):
            m.forward(x)
            ms, flops = m.last_forward()
            best = ms if best is None else min(best, ms)
        return best, flops

    best, flops = timed(fused)
    chain = timed(False)[0] if (chain_too and fused) else None
    m.close()
    peak, kind = tensor_peak()
    tf = flops / (best / 1e3) / 1e12
    M = (rows + 127) // 128 * 128
    # HBM bytes: the fused kernel reads the BF16 input and writes the FP32
    # output; the chain also writes and re-reads every BF16 hidden activation
    fused_bytes = M * (48 * 2 + 48 * 4)
    chain_bytes = M * (48 * 2 + 256 * 2) + 2 * M * (256 * 2 + 256 * 2) + M * (256 * 2 + 48 * 4)
    hbm = fused_bytes if fused else chain_bytes
    hpeak, hkind = peaks()
    out = {"workload": f"surrogate ranking: {rows} candidates through 38-256-256-256-33 (padded 48 / 48)",
           "kernel": "fused four-layer kernel" if fused else "layer-by-layer GEMM chain",
           "ms": best, "flops": flops, "tflops": tf,
           "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "unit": "TFLOP/s", "frac": tf / peak,
                        "peak_source": kind},
           "hbm": {"algorithmic_bytes": hbm, "achieved_gbs": hbm / (best / 1e3) / 1e9,
                   "frac": hbm / (best / 1e3) / 1e9 / hpeak}}
    if chain is not None:
        out["layer_chain"] = {"ms": chain, "tflops": flops / (chain / 1e3) / 1e12, "speedup_fused": chain / best}
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int = 0):
        self.path = tempfile.mktemp(prefix="felis_clocks_", suffix=".csv")
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_config(name: str, slices: int | None = None, grid: int | None = None, world: int = 1, rank: int = 0):
    """The workload's input file parsed for `rank` of `world` slice blocks
    (one block: the whole bunch)."""
    import felis_b200 as fb
    from felis_b200 import workloads

    d = tempfile.mkdtemp(prefix="felis_bench_")
    kw = dict(workloads.WORKLOADS[name])
    if slices and name == "sase":
        kw["slices"] = slices
    if grid:
        kw["nx"] = grid
    return fb.Config(workloads.write_input(os.path.join(d, f"{name}.inp"), **kw), world, rank)


def workload_config(name: str, p, P: int, W: int, K: int, world: int, precision: str) -> dict:
    """The line's `config`: the workload, its sizes and the timed iterations."""
    what = (f"{name}: {precision} time-dependent SASE, {p.slice_n} slices x {P // p.slice_n} particles, "
            f"{p.nx}x{p.ny} grid, H={p.num_harmony}" if name == "sase"
            else f"{name}: {precision} static, {P} particles, {p.nx}x{p.ny} grid")
    return {"workload": what, "slices": p.slice_n, "particles": P, "grid": [p.nx, p.ny], "harmonics": p.num_harmony,
            "iterations": [W, W + K], "l2": "inputs larger than L2 (particles 403 MB, field 171 MB per pol)",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"}


def reference_config(name: str) -> dict:
    """The `config` of the reference arm's line, from the workload table
    alone (no product code is loaded on that arm)."""
    wl = _workloads_module()
    kw = dict(wl.WORKLOADS[name])
    n = kw.get("nx", 101) + 1
    if name == "sase":
        S = kw.get("slices", 1024)
        P = S * kw.get("beamlets", 2048) * kw.get("per_beamlet", 4)
        what = (f"{name}: FP64 time-dependent SASE, {S} slices x {P // S} particles, {n}x{n} grid, H=1 "
                f"(the reference's own CPU step loop; same workload as the GPU arm's line)")
    else:
        S, P = 1, kw.get("beamlets", 2048) * kw.get("per_beamlet", 4)
        what = f"{name}: FP64 static, {P} particles, {n}x{n} grid (the reference's own CPU step loop)"
    return {"workload": what, "slices": S, "particles": P, "grid": [n, n], "harmonics": 1,
            "parallelism": "host cores, one rank of the reference's slice decomposition per core"}


def make_workload(name: str, rank: int = 0, slices: int | None = None, grid: int | None = None):
    cfg = make_config(name, slices, grid)
    beam = cfg.load_beam(0, seed=2 if name == "sase" else 1)
    fields = [cfg.load_seed(h) for h in range(cfg.params.num_harmony)]
    return cfg, beam, fields


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None, 0, 1
    import datetime

    import torch
    import torch.distributed as dist

    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return dist, rank, world


def max_over_ranks(dist, v: float) -> float:
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def _workloads_module():
    """felis_b200/workloads.py loaded on its own: the reference arm writes the
    workload's input file without importing the package (which would load
    the product library)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("felis_workloads", os.path.join(ROOT, "felis_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_cpu(name: str, warmup: int, steps: int, procs: int) -> tuple[float, str, str]:
    """The reference's own step loop on the host cores: oracle/_ref/
    felis_ref_fast (the reference's unmodified sources, built with its
    makefile's flags) from the workload's input file, loading its beam with
    its own loader.  `procs` processes each play one rank of the reference's
    slice decomposition (boundary.cpp:33-46; loadBeam's per-rank Halton skip,
    loadBeam.cpp:78-91), so each computes exactly its rank's share of every
    step; the one-plane halo message of fieldShareZ.cpp:39-78 does not cross
    processes (the stand-in MPI drops it).  Value: all ranks' particles x
    timed iterations / the slowest rank's loop time.  Returns (value,
    sample description, kind)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun
    from concurrent.futures import ThreadPoolExecutor

    wl = _workloads_module()
    kw = dict(wl.WORKLOADS[name])
    d = tempfile.mkdtemp(prefix="felis_ref_bench_")
    path = wl.write_input(os.path.join(d, f"{name}.inp"), **kw)
    with open(path) as f:
        slices = 1 if "mode=Static" in f.read() else kw.get("slices", 1024)
    procs = max(1, min(procs, slices))
    seed = 2 if name == "sase" else 1

    def one(rank):
        return refrun.run(path, it1=warmup + steps, time_warmup=warmup, final=False, variant="fast", seed=seed,
                          ranks=(procs, rank), timeout=1800)["timing"]

    with ThreadPoolExecutor(max_workers=procs) as ex:
        timings = list(ex.map(one, range(procs)))
    secs = max(t["seconds"] for t in timings)
    particles = sum(t["particles"] for t in timings)
    value = particles * steps / secs
    sample = (f"the whole workload ({int(particles)} particles, {slices} slices), iterations {warmup}..{warmup + steps - 1} "
              f"after {warmup} untimed, {secs:.2f} s timed (slowest of {procs} rank processes, one per host core); "
              f"the reference's own loader, tables and step loop (oracle/_ref/felis_ref_fast: unmodified sources, "
              f"makefile flags with -march=x86-64-v3)")
    return value, sample, "reference"


def cpu_sample(name: str, steps: int, warmup: int, target_s: float, threads: int):
    """The CPU baseline: the reference's own loop (reference_cpu) when
    oracle/_ref is built, else the restatement (reference compiler flags) on
    a slice subset of the workload; returns (particle-steps/s, description,
    kind)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun

    if refrun.available("fast"):
        return reference_cpu(name, min(warmup, 3), max(1, min(steps, 20)), threads)
    import oracle

    import felis_b200 as fb
    from felis_b200 import workloads

    out_dir = tempfile.mkdtemp(prefix="felis_oracle_")
    variant = "fast"
    try:
        oracle.build("fast", out_dir)
    except Exception:
        variant, out_dir = "strict", None
    base = dict(workloads.WORKLOADS[name])
    total_slices = 1024 if name == "sase" else 1

    def run(slices: int, nsteps: int):
        kw = dict(base)
        if name == "sase":
            kw["slices"] = slices
        d = tempfile.mkdtemp(prefix="felis_cpu_")
        cfg = fb.Config(workloads.write_input(os.path.join(d, "s.inp"), **kw))
        b = cfg.load_beam(0, seed=2 if name == "sase" else 1)
        o = oracle.Oracle(cfg.params, threads=threads, variant=variant, out_dir=out_dir)
        o.set_particles(0, b["x"], b["y"], b["px"], b["py"], b["theta"], b["gamma"], b["offsets"], b["weights"])
        for hh in range(cfg.params.num_harmony):
            ux, uy = cfg.load_seed(hh)
            o.set_field(hh, 0, ux)
            o.set_field(hh, 1, uy)
        o.run(0, warmup, diagnostics=True)
        t0 = time.perf_counter()
        o.run(warmup, warmup + nsteps, diagnostics=True)
        dt = time.perf_counter() - t0
        return int(b["offsets"][-1]), dt, cfg.params

    # calibrate on one slice per thread for one iteration, then size the
    # sample so the timed part takes about target_s seconds
    probe = min(total_slices, threads)
    n, dt, p = run(probe, 1)
    rate = n / max(dt, 1e-6)
    per_slice = max(n // probe, 1)
    nsteps = max(1, min(steps, 3))
    slices = total_slices if name != "sase" else int(min(total_slices, max(probe, target_s * rate / (per_slice * nsteps))))
    n, dt, p = run(slices, nsteps)
    value = n * nsteps / dt
    sample = (f"{slices} of {total_slices} slices x {n // max(slices, 1)} particles, iterations "
              f"{warmup}..{warmup + nsteps - 1} after {warmup} untimed, {dt:.1f} s timed on {threads} threads; "
              f"CPU restatement, build '{variant}' (reference compiler flags)")
    return value, sample, "port"


def run_sharded(args, dist, rank, world):
    """One FP64 run of the workload with its slices split into contiguous
    blocks, one per rank (boundary.cpp:33-46; strong scaling: the bunch is
    fixed, each rank steps 1/N of it).  After every shifted iteration the
    slipping slice's planes go to the next rank in device memory
    (fieldShareZ.cpp:39-78: NCCL send / receive on the handle's stream,
    felis_b200.shard), rank 0 takes zeros.  Each step is one drop-in
    felis_step call; the diagnostics stay on the device in the timed region
    and are reduced over the ranks afterwards (updateTotalEnergy.cpp:56-68)."""
    import numpy as np
    import torch

    import felis_b200 as fb
    from felis_b200 import shard

    cfg = make_config(args.workload, args.slices, args.grid, world, rank)
    p = cfg.params
    beam = cfg.load_beam(0, seed=2 if args.workload == "sase" else 1)
    fields = [cfg.load_seed(h) for h in range(p.num_harmony)]
    P = int(beam["offsets"][-1])
    h = fb.Handle(p)
    h.upload_particles(0, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"],
                       beam["offsets"], beam["weights"])
    for hh, (ux, uy) in enumerate(fields):
        h.upload_field(hh, 0, ux)
        h.upload_field(hh, 1, uy)
    del beam, fields
    eng = shard.GpuEngine(h)
    loop = shard.ShardedLoop(eng, dist, rank, world) if dist is not None else None
    st = eng.stream()

    def advance(it0, it1):
        for it in range(it0, it1):
            if eng.step(it):
                if loop is not None:
                    loop.exchange()
                else:
                    shard.exchange_in_process([eng])  # one block: the first slice takes zeros

    W, K = args.warmup, args.steps
    advance(0, W)
    h.sync()
    h.profile(True, max_launches=16 * K + 64)  # launch counts of the timed region
    barrier(dist)
    torch.cuda.synchronize()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    advance(W, W + K)
    e1.record(st)
    h.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(dist)
    ms = max_over_ranks(dist, e0.elapsed_time(e1))
    e, _, _ = h.diagnostics(W, W + K)
    total = np.array([float(P)] + list(e[-1]), dtype=np.float64)
    if dist is not None:
        t = torch.from_numpy(total).cuda()
        dist.all_reduce(t)
        total = t.cpu().numpy()
    particles = int(total[0])
    value = particles * K / (ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded beam loader of the reference input format, per slice block)",
        "config": {"workload": f"{args.workload}: FP64 time-dependent SASE, {p.global_slice_n} slices split into "
                               f"{world} blocks, {particles} particles, {p.nx}x{p.ny} grid, H={p.num_harmony}",
                   "slices": p.global_slice_n, "particles": particles, "grid": [p.nx, p.ny],
                   "iterations": [W, W + K], "parallelism": f"slice blocks x{world}",
                   "exchange": "device memory, NCCL send/recv on the library stream" if world > 1 else "none",
                   "l2": "inputs larger than L2"},
        "final_power_units": float(total[1]), "clocks": clk, "gpu_launches": h.kernel_stats(-1)[0],
        "cpu_baseline": None, "e2e": None,
    }
    h.close()
    return line


def run_felis(args, dist, rank, world):
    import numpy as np

    import felis_b200 as fb

    cfg, beam, fields = make_workload(args.workload, rank, args.slices, args.grid)
    p = cfg.params
    P = int(beam["offsets"][-1])
    cells = p.slice_n * p.nx * p.ny * 2 * p.num_harmony
    h = fb.Handle(p)
    h.upload_particles(0, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"],
                       beam["offsets"], beam["weights"])
    for hh, (ux, uy) in enumerate(fields):
        h.upload_field(hh, 0, ux)
        h.upload_field(hh, 1, uy)
    W, K = args.warmup, args.steps
    h.run(0, W)
    h.sync()
    # ---- timed region: K iterations from one graph, events on the library stream ----
    h.profile(True, max_launches=16 * K + 64)
    barrier(dist)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    time.sleep(0.3)
    h.run(W, W + K)
    h.sync()
    ms = h.last_run_ms()
    clk = clocks.stop()
    barrier(dist)
    ms = max_over_ranks(dist, ms)
    sec = ms / 1e3
    kinds = {}
    for name, k in fb.KERNEL_KINDS.items():
        n, t = h.kernel_stats(k)
        kinds[name] = {"launches": n, "ms": t}
    launches, _ = h.kernel_stats(-1)
    e, tw, bf = h.diagnostics(W, W + K)
    value = P * K * world / sec
    adi_cells = cells * K * world / sec
    # dominant kernel roofline (HBM): algorithmic bytes per launch / mean launch time
    dom = max(kinds, key=lambda k: kinds[k]["ms"])
    bytes_per_launch = {"particles": P * BYTES_PARTICLE_STEP, "adi": cells * BYTES_ADI_CELL,
                        "deposit": P * 4 + p.slice_n * p.nx * p.ny * 2 * p.num_harmony * 16,
                        "reduce": 0, "shift": 0}
    peak, peak_kind = peaks()
    kd = kinds[dom]
    avg_ms = kd["ms"] / max(kd["launches"], 1)
    achieved = bytes_per_launch[dom] / (avg_ms / 1e3) / 1e9 if avg_ms > 0 else 0.0
    step_bytes = P * BYTES_PARTICLE_STEP + cells * BYTES_ADI_CELL
    traffic = None
    prof_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof_path):
        try:
            with open(prof_path) as f:
                traffic = json.load(f).get(args.workload, {}).get(dom)
        except Exception:
            traffic = None
    # ---- end to end through the C ABI with host buffers ----
    e2e = run_e2e(args, cfg, beam, fields, dist)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded beam loader of the reference input format)",
        "config": workload_config(args.workload, p, P, W, K, world, "FP64"),
        "adi_cells_per_s": adi_cells,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "bytes_per_launch": bytes_per_launch[dom], "mean_launch_ms": avg_ms},
        "step_roofline": {"algorithmic_bytes": step_bytes, "achieved_gbs": step_bytes / (ms / K / 1e3) / 1e9,
                          "frac": step_bytes / (ms / K / 1e3) / 1e9 / peak},
        "kernels": kinds,
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": e2e,
        "final_power_units": float(e[-1, 0]),
        "_energy": h.diagnostics(0, W + K + 1)[0],
    }
    h.close()
    return line


BYTES_PARTICLE_STEP_MIXED = 56  # read + write of 5 x 4 B + theta 8 B
BYTES_ADI_CELL_MIXED = 16       # read + write one FP32 complex cell


def _batch_upload(b, k, beam, fields):
    """Particles (host arrays or device tensors) and, unless None (a run
    without seed laser: the engine's field starts at zero), the seed field."""
    b.upload_particles(k, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"],
                       beam["offsets"], beam["weights"])
    for hh, (ux, uy) in enumerate(fields or []):
        b.upload_field(k, hh, 0, ux)
        b.upload_field(k, hh, 1, uy)


def batch_kernels(b):
    import felis_b200 as fb

    out = {}
    for name, k in fb.BATCH_KERNEL_KINDS.items():
        n, t = b.kernel_stats(k)
        out[name] = {"launches": n, "ms": t}
    return out


def run_mixed(args, cfg, beam, fields, dist, world, fp64_energy):
    """The workload through the mixed-precision engine: tuned launch shape,
    W warm-up iterations, K timed iterations from one graph; power error
    against the FP64 plain run of the same iterations."""
    import numpy as np

    import felis_b200 as fb
    from felis_b200 import analysis

    p = cfg.params
    P = int(beam["offsets"][-1])
    cells = p.slice_n * p.nx * p.ny * 2 * p.num_harmony
    b = fb.Batch([p])
    _batch_upload(b, 0, beam, fields)
    W, K = args.warmup, args.steps
    # the tuner advances the run; start it over for the measured iterations
    b.tune(0, 2)
    b.close()
    b = fb.Batch([p])
    _batch_upload(b, 0, beam, fields)
    b.run(0, W)
    b.profile(True, max_launches=8 * K + 64)
    barrier(dist)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    time.sleep(0.3)
    b.run(W, W + K)
    ms = b.last_run_ms()
    clk = clocks.stop()
    barrier(dist)
    ms = max_over_ranks(dist, ms)
    kinds = batch_kernels(b)
    launches, _ = b.kernel_stats(-1)
    e, tw, bf = b.diagnostics(0, 0, W + K + 1)
    P32 = analysis.output_power(e)
    P64 = analysis.output_power(fp64_energy)
    ok = P64 > 0
    rel = np.abs(P32[ok] - P64[ok]) / P64[ok]
    sec = ms / 1e3
    peak, peak_kind = peaks()
    bytes_per_launch = {"push": P * BYTES_PARTICLE_STEP_MIXED, "adi": cells * BYTES_ADI_CELL_MIXED, "reduce": 0}
    dom = max(("push", "adi"), key=lambda k: kinds[k]["ms"])
    kd = kinds[dom]
    avg_ms = kd["ms"] / max(kd["launches"], 1)
    achieved = bytes_per_launch[dom] / (avg_ms / 1e3) / 1e9 if avg_ms > 0 else 0.0
    step_bytes = P * BYTES_PARTICLE_STEP_MIXED + cells * BYTES_ADI_CELL_MIXED
    traffic = None
    prof_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof_path):
        try:
            with open(prof_path) as f:
                traffic = json.load(f).get(args.workload + "_mixed", {}).get(dom)
        except Exception:
            traffic = None
    box, adi_ctas = b.launch()
    res = {
        "value": P * K * world / sec, "ms_per_step": ms / K, "adi_cells_per_s": cells * K * world / sec,
        "launch": {"push_box_cells": box, "adi_ctas_per_sm": adi_ctas},
        "power_error": {"max_rel": float(rel.max()) if rel.size else None,
                        "final_rel": float(rel[-1]) if rel.size else None,
                        "iterations": [0, W + K], "reference": "FP64 plain GPU path, same initial state"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "bytes_per_launch": bytes_per_launch[dom], "mean_launch_ms": avg_ms},
        "step_roofline": {"algorithmic_bytes": step_bytes, "achieved_gbs": step_bytes / (ms / K / 1e3) / 1e9,
                          "frac": step_bytes / (ms / K / 1e3) / 1e9 / peak},
        "kernels": kinds, "gpu_launches": launches, "clocks": clk,
    }
    b.close()
    return res


def run_mixed_e2e(args, cfg, beam, fields, dist):
    """The mixed engine end to end through the C ABI: upload from pinned host
    buffers (FP64, converted by the library), K iterations, the per-iteration
    diagnostics read back, the final particles downloaded into pinned host
    buffers."""
    import numpy as np

    import felis_b200 as fb

    try:
        import torch

        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.complex128, pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()
    except Exception:
        def pinned(a):
            return np.array(a)

    p = cfg.params
    host = {k: pinned(np.asarray(beam[k])) for k in ("x", "y", "px", "py", "theta", "gamma")}
    hf = [(pinned(ux), pinned(uy)) for ux, uy in fields]
    K = max(1, min(args.steps, args.e2e_steps))
    P = int(beam["offsets"][-1])
    # the result lands in pinned host buffers, allocated (and touched) before the timing
    res = {k: pinned(np.zeros(P)) for k in ("x", "y", "px", "py", "theta", "gamma")}
    b = fb.Batch([p])
    barrier(dist)
    t0 = time.perf_counter()
    b.upload_particles(0, host["x"], host["y"], host["px"], host["py"], host["theta"], host["gamma"],
                       beam["offsets"], beam["weights"])
    for hh, (ux, uy) in enumerate(hf):
        b.upload_field(0, hh, 0, ux)
        b.upload_field(0, hh, 1, uy)
    b.run(0, K)
    b.diagnostics(0, 0, K + 1)
    b.download_particles(0, out=res)
    dt = time.perf_counter() - t0
    barrier(dist)
    dt = max_over_ranks(dist, dt)
    world = 1 if dist is None else dist.get_world_size()
    h2d = 6 * P * 8 + sum(2 * a.nbytes for a, _ in hf)
    d2h = (K + 1) * (2 * p.num_harmony + 6 + 2 * p.num_harmony) * 8 + 6 * P * 8
    b.close()
    return {"value": P * K * world / dt, "unit": UNIT, "steps": K, "seconds": dt,
            "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
            "api": "felis_batch_upload_* + felis_batch_run + felis_batch_get_diagnostics + "
                   "felis_batch_download_particles"}


def run_ensemble(args, dist, world):
    """The 96-instance batched ensemble: aggregate throughput, and the power
    error of every instance against an FP64 plain run of the same
    iterations."""
    import numpy as np

    import felis_b200 as fb
    from felis_b200 import analysis, workloads

    spec = workloads.ensemble(args.ensemble)
    d = tempfile.mkdtemp(prefix="felis_ens_")
    cfgs = []
    for k, kw in enumerate(spec):
        kw = dict(kw)
        seed = kw.pop("beam_seed")
        kw["total_length"] = 40.0
        cfgs.append((fb.Config(workloads.write_input(os.path.join(d, f"i{k}.inp"), **kw)), seed))
    t_setup = time.perf_counter()
    b = fb.Batch([c.params for c, _ in cfgs])
    P = 0
    cells = 0
    # beams from the device loader; no seed laser, so the fields start at zero
    for k, (c, seed) in enumerate(cfgs):
        beam = c.load_beam_device(0, seed=seed)
        _batch_upload(b, k, beam, None)
        P += int(beam["offsets"][-1])
        cells += c.params.slice_n * c.params.nx * c.params.ny * 2 * c.params.num_harmony
        del beam
    t_setup = time.perf_counter() - t_setup
    W, K = args.warmup, args.ensemble_steps
    nxt = b.tune(0, 1)
    b.run(nxt, nxt + W)
    b.profile(True, max_launches=8 * K + 64)
    barrier(dist)
    i0 = nxt + W
    b.run(i0, i0 + K)
    ms = max_over_ranks(dist, b.last_run_ms())
    barrier(dist)
    kinds = batch_kernels(b)
    launches, _ = b.kernel_stats(-1)
    # per-instance power error, every instance: the same instance from the same
    # initial state through the FP64 plain path for the same iterations
    errs = []
    for k, (c, seed) in enumerate(cfgs):
        beam = c.load_beam_device(0, seed=seed)  # the instance's initial state
        h = fb.Handle(c.params)
        h.upload_particles(0, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"],
                           beam["offsets"], beam["weights"])
        del beam
        h.run(0, i0 + K)
        P64 = analysis.output_power(h.diagnostics(0, i0 + K + 1)[0])
        P32 = analysis.output_power(b.diagnostics(k, 0, i0 + K + 1)[0])
        ok = P64 > 0
        rel = np.abs(P32[ok] - P64[ok]) / P64[ok]
        errs.append((float(rel.max()), k, c.params.slice_n, c.params.nx))
        h.close()
    worst = max(errs)
    box, adi_ctas = b.launch()
    res = {
        "workload": f"{len(spec)} SASE instances (shot noise, no seed laser), slices in {{128..2048}}, "
                    f"grids {{66, 102, 152}}, 4096 particles per slice, 2-4 kA, spread 0.5-2e-4, mixed precision; "
                    f"beams from the device loader",
        "value": P * K * world / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / K,
        "adi_cells_per_s": cells * K * world / (ms / 1e3), "particles": P, "cells": cells,
        "steps": K, "iterations": [i0, i0 + K], "setup_s": t_setup,
        "launch": {"push_box_cells": box, "adi_ctas_per_sm": adi_ctas},
        "kernels": kinds, "gpu_launches": launches,
        "power_error_vs_fp64": {
            "instances": len(errs), "what": "per instance, the largest relative power error over iterations "
                                            f"0..{i0 + K} against the FP64 plain path from the same initial state",
            "max": worst[0], "median": float(np.median([e[0] for e in errs])),
            "worst_instance": {"index": worst[1], "slices": worst[2], "grid": worst[3]},
            "per_instance": [e[0] for e in sorted(errs, key=lambda e: e[1])]},
    }
    b.close()
    return res


def run_config3(args, dist, world):
    """A timed prefix of the mixed-precision long run (the Gaussian-current
    tapered SASE workload "gaussian_taper": 4096 slices, QuadPolar with
    polarity 0.5, harmonics 1 and 3, copper AC wake, 152 x 152 grid) through
    the FP64 plain path and the mixed engine from the same initial state:
    W untimed iterations, K timed from one graph each, the power error of
    every iteration 0..W+K per harmonic.  Early iterations run faster per
    step than the run's average (the beam and its deposit box grow along
    the undulator; the whole 60 m is measured by python -m
    felis_b200.longrun)."""
    import numpy as np

    import felis_b200 as fb
    from felis_b200 import analysis, longrun

    t0 = time.perf_counter()
    cfg, beam, fields, kw = longrun.prepare("gaussian_taper")
    p = cfg.params
    P = int(beam["offsets"][-1])
    cells = p.slice_n * p.nx * p.ny * 2 * p.num_harmony
    setup_s = time.perf_counter() - t0
    W, K = args.warmup, args.config3_steps
    peak, peak_kind = peaks()

    def timed(obj, stats_kinds, run, diag):
        run(0, W)
        obj.profile(True, max_launches=16 * K + 64)
        barrier(dist)
        run(W, W + K)
        ms = max_over_ranks(dist, obj.last_run_ms())
        kinds = {}
        for name, k in stats_kinds.items():
            n, t = obj.kernel_stats(k)
            kinds[name] = {"launches": n, "ms": t}
        return ms, kinds, diag(W + K + 1)

    h = fb.Handle(p)
    h.upload_particles(0, *(beam[k] for k in ("x", "y", "px", "py", "theta", "gamma")), beam["offsets"], beam["weights"])
    ms64, k64, e64 = timed(h, fb.KERNEL_KINDS, h.run, lambda n: h.diagnostics(0, n)[0])
    launches64, _ = h.kernel_stats(-1)
    h.close()
    b = fb.Batch([p])
    _batch_upload(b, 0, beam, fields)
    b.tune(0, 2)
    launch = b.launch()
    b.close()
    b = fb.Batch([p])
    b.set_launch(*launch)
    _batch_upload(b, 0, beam, fields)
    ms32, k32, e32 = timed(b, fb.BATCH_KERNEL_KINDS, b.run, lambda n: b.diagnostics(0, 0, n)[0])
    launches32, _ = b.kernel_stats(-1)
    b.close()
    errs = {}
    for hidx in range(p.num_harmony):
        P64, P32 = analysis.output_power(e64, hidx), analysis.output_power(e32, hidx)
        ok = P64 > 0
        rel = np.abs(P32[ok] - P64[ok]) / P64[ok]
        errs[f"H{p.harmony[hidx]}"] = {"max_rel": float(rel.max()) if rel.size else None,
                                       "final_rel": float(rel[-1]) if rel.size else None}
    dom = max(("push", "adi"), key=lambda k: k32[k]["ms"])
    kd = k32[dom]
    avg_ms = kd["ms"] / max(kd["launches"], 1)
    bpl = {"push": P * BYTES_PARTICLE_STEP_MIXED, "adi": cells * BYTES_ADI_CELL_MIXED}[dom]
    achieved = bpl / (avg_ms / 1e3) / 1e9 if avg_ms > 0 else 0.0
    return {
        "workload": f"gaussian_taper: {p.slice_n} slices, Gaussian current (rms 600 slices, peak 4 kA, "
                    f"{P} particles), QuadPolar polarity 0.5, harmonics 1 and 3, copper AC wake, "
                    f"{p.nx}x{p.ny} grid, linear taper -1 %; timed prefix of the 60 m run",
        "particles": P, "cells_per_step": cells, "iterations": [W, W + K], "setup_s": setup_s,
        "fp64": {"ms_per_step": ms64 / K, "value": P * K * world / (ms64 / 1e3),
                 "adi_cells_per_s": cells * K * world / (ms64 / 1e3), "kernels": k64, "gpu_launches": launches64},
        "mixed": {"ms_per_step": ms32 / K, "value": P * K * world / (ms32 / 1e3),
                  "adi_cells_per_s": cells * K * world / (ms32 / 1e3), "kernels": k32, "gpu_launches": launches32,
                  "launch": {"push_box_cells": launch[0], "adi_ctas_per_sm": launch[1]},
                  "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                               "frac": achieved / peak, "peak_source": peak_kind, "bytes_per_launch": bpl,
                               "mean_launch_ms": avg_ms}},
        "speedup_mixed_vs_fp64": ms64 / ms32,
        "power_error_vs_fp64": errs,
    }


def run_e2e(args, cfg, beam, fields, dist):
    """Upload from pinned host memory, K iterations through felis_step with
    each iteration's diagnostics read back, final particles downloaded."""
    import numpy as np

    import felis_b200 as fb

    try:
        import torch

        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.complex128, pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()
    except Exception:
        def pinned(a):
            return np.array(a)

    p = cfg.params
    host = {k: pinned(np.asarray(beam[k])) for k in ("x", "y", "px", "py", "theta", "gamma")}
    hf = [(pinned(ux), pinned(uy)) for ux, uy in fields]
    res = {k: pinned(np.zeros(int(beam["offsets"][-1]))) for k in ("x", "y", "px", "py", "theta", "gamma")}
    K = max(1, min(args.steps, args.e2e_steps))
    P = int(beam["offsets"][-1])
    h = fb.Handle(p)
    barrier(dist)
    t0 = time.perf_counter()
    h.upload_particles(0, host["x"], host["y"], host["px"], host["py"], host["theta"], host["gamma"],
                       beam["offsets"], beam["weights"])
    for hh, (ux, uy) in enumerate(hf):
        h.upload_field(hh, 0, ux)
        h.upload_field(hh, 1, uy)
    for it in range(K):
        h.step(it)
        h.diagnostics(it, it + 1)
    out = h.download_particles(0, out=res)
    dt = time.perf_counter() - t0
    barrier(dist)
    dt = max_over_ranks(dist, dt)
    world = 1 if dist is None else dist.get_world_size()
    h2d = 6 * P * 8 + sum(2 * a.nbytes for a, _ in hf)
    d2h = K * (2 * p.num_harmony + 6 * p.num_species + 2 * p.num_harmony) * 8 + 6 * P * 8
    h.close()
    return {"value": P * K * world / dt, "unit": UNIT, "steps": K, "seconds": dt,
            "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
            "api": "felis_upload_* + felis_step + felis_get_diagnostics per iteration + felis_download_particles"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["felis", "reference"], default="felis")
    ap.add_argument("--workload", choices=["sase", "static"], default="sase")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--slices", type=int, default=None, help="smaller sase bunch (profiling captures)")
    ap.add_argument("--grid", type=int, default=None, help="grid key nx = ny of the workload (profiling captures)")
    ap.add_argument("--ensemble", type=int, default=96, help="instances of the batched ensemble (0: skip)")
    ap.add_argument("--ensemble-steps", type=int, default=10)
    ap.add_argument("--surrogate-rows", type=int, default=1_000_000,
                    help="candidates of the timed surrogate ranking (0: skip)")
    ap.add_argument("--config3-steps", type=int, default=20,
                    help="timed iterations of the Gaussian-current tapered run (0: skip)")
    ap.add_argument("--fp64-only", action="store_true", help="the FP64 plain path alone (profiling captures)")
    ap.add_argument("--sharded", action="store_true",
                    help="one FP64 run with its slices split over the ranks (strong scaling, device halo exchange)")
    ap.add_argument("--surrogate-chain", action="store_true",
                    help="with --surrogate-only: the layer-by-layer GEMM chain instead of the fused kernel")
    ap.add_argument("--surrogate-only", action="store_true",
                    help="the surrogate ranking GEMM chain alone (profiling captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        cores = host_cores()
        value, sample, kind = cpu_sample(args.workload, args.steps, args.warmup, 20.0, cores)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "higher_is_better": True,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "dtype": "f64",
            "config": reference_config(args.workload),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }), flush=True)
        return

    if args.surrogate_only:
        print(json.dumps(run_surrogate_gemm(args.surrogate_rows, chain_too=False, fused=not args.surrogate_chain)),
              flush=True)
        return
    dist, rank, world = dist_init()
    if args.sharded:
        line = run_sharded(args, dist, rank, world)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    line = run_felis(args, dist, rank, world)
    if not args.fp64_only:
        cfg, beam, fields = make_workload(args.workload, rank, args.slices, args.grid)
        fp64 = dict(line)
        e64 = fp64.pop("_energy")
        mixed = run_mixed(args, cfg, beam, fields, dist, world, e64)
        e2e = run_mixed_e2e(args, cfg, beam, fields, dist)
        del beam, fields
        ens = run_ensemble(args, dist, world) if args.ensemble > 0 else None
        c3 = run_config3(args, dist, world) if args.config3_steps > 0 else None
        sg = run_surrogate_gemm(args.surrogate_rows) if args.surrogate_rows > 0 else None
        for k in ("metric", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline",
                  "data", "cpu_baseline"):
            fp64.pop(k, None)
        cfg_line = dict(line["config"])
        cfg_line["workload"] = cfg_line["workload"].replace("FP64 ", "mixed-precision ")
        line = {
            "metric": METRIC, "value": mixed["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mixed["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (theta, lattice, reductions f64)",
            "data": line["data"], "config": cfg_line,
            "adi_cells_per_s": mixed["adi_cells_per_s"],
            "speedup_vs_fp64_plain": mixed["value"] / fp64["value"],
            "power_error_vs_fp64": mixed["power_error"],
            "roofline": mixed["roofline"], "step_roofline": mixed["step_roofline"],
            "kernels": mixed["kernels"], "gpu_launches": mixed["gpu_launches"], "clocks": mixed["clocks"],
            "launch": mixed["launch"], "e2e": e2e, "fp64_plain": fp64, "ensemble": ens, "config3": c3,
            "surrogate_gemm": sg,
        }
    else:
        line.pop("_energy", None)
    if rank == 0:
        if args.no_cpu_baseline or world > 1:  # the host baseline is timed once, at one GPU
            line["cpu_baseline"] = None
        else:
            cores = host_cores()
            v, sample, kind = cpu_sample(args.workload, 5, 2, args.cpu_seconds, cores)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
            if "fp64_plain" in line:
                fp = line["fp64_plain"]
                line["precision_matched"] = {
                    "what": "FP64 against FP64: the GPU's FP64 plain path over the reference's own CPU loop "
                            "(cpu_baseline), device-timed and end to end",
                    "fp64_gpu_value": fp["value"], "fp64_gpu_e2e": fp["e2e"]["value"], "cpu_reference_fp64": v,
                    "ratio_device": fp["value"] / v, "ratio_e2e": fp["e2e"]["value"] / v,
                    "mixed_over_cpu_reference_fp64": line["value"] / v}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
