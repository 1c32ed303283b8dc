#!/usr/bin/env python
"""P3M bodies*steps/s on B200 — the benchmark of this library.

One step = one gravity-only P3M leapfrog step of the workload
(GravityPipeline.step without collisions): Morton reorder every second step,
half kick + drift, cell-key sort and lists, CIC deposit, real FFT with the
Green's multiply, inverse, interpolation + short range + half kick.

Default workload (N=1): the precision form at scale, 8,000,000 bodies from a
4096x2048 lattice displaced by a Gaussian random field (P(k) ~ k^-2,
displacement RMS 3 cells, seed 7) on a 4096x2048 torus, int64 fixed-point
deposit, FP32 FFT and forces. Beside it (`plain_form`): 400,000 bodies in two
projected Plummer spheres inside walls, physical grid 512x256 (Hockney FFT
mesh 1024x512), the reference's uint32 deposit. L2 is flushed (a 256 MiB
write) before every timed step, outside the step's events (the 400k state
fits in the 126 MB L2; the 8M state does not). Without flags, W = 5 warm-up
and K = 45 timed steps: the 50 steps of the precision-form configuration
(the lattice clusters as it evolves, so longer runs time other states).
Before timing, the library's autotuner (p3m_autotune) picks the launch
shapes and puts the state back; the line reports its choice.

Printed (rank 0, one JSON line):
  value     bodies*steps/s from CUDA events around each step, state resident
            in HBM, summed over the K timed steps, max over ranks.
  e2e       the same through the public API with host buffers: every step
            uploads the body state (positions, velocities) from page-locked
            memory, steps, and reads the bodies back (host wall clock over
            all steps, up to the last download). `value` is the pipelined
            form (p3m_step_io: step k+1's upload and step k's download run
            on the copy engines while the steps compute); `serial_value`
            waits for each copy before the next call. The per-body
            materials are static and uploaded once, before timing, as the
            reference uploads them when it seeds bodies.
  roofline  the dominant stage's algorithmic bytes / its event-timed average
            duration, against the measured HBM copy bandwidth; every stage's
            fraction is in `stages`, the deposit's and the kick's also in
            `roofline_hbm_stages`. The short range is bound by its exp2 and
            reciprocal operations, not by DRAM: `roofline.xu` gives that
            floor (the MUFU unit's rate at the sampled SM clock) and the
            fraction of it reached.
  force_rms_err_vs_fp64_by_form  RMS force error against the FP64 direct sum
            on one seeded 4096-body subsample for the int64 form, the uint32
            form and the CPU oracle's FP32 path.
  cpu_baseline  the CPU oracle (the C++ restatement of the reference's
            shaders) on this host's cores, on a bounded sample.

`--impl reference` times the reference's CPU path, i.e. the oracle port (the
reference has no CPU implementation and its GLSL cannot run here), with all
host threads, on the same workload and metric.

Multi-GPU (torchrun): replicas only. Every rank runs its own copy of the
workload; value = all bodies*steps / the slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

METRIC = ("P3M bodies·steps/s on 1 B200 (plain vs chosen form) at stated force RMS err "
          "vs FP64")
UNIT = "bodies*steps/s"
L2_FLUSH_BYTES = 256 << 20
FORCE_SAMPLE = 4096


# ----------------------------------------------------------------- workloads
def make_workload(name: str, bodies: int | None = None, grid: str | None = None,
                  sims: int | None = None):
    """A named workload at its stated size, or with `bodies` / `grid` (WxH)
    overridden: the smaller cases the committed Nsight Compute captures run."""
    from gravity_b200 import scenarios

    g = tuple(int(v) for v in grid.split("x")) if grid else None
    if name == "plummer_walls":
        return scenarios.plummer_walls(**({"n": bodies} if bodies else {}))
    if name == "uniform_torus":
        return scenarios.uniform_torus(**({"n": bodies} if bodies else {}))
    if name in ("lattice_scale", "lattice_scale_u32"):
        from gravity_b200 import _abi
        kw = {}
        if bodies:
            kw["n"] = bodies
        if g:
            kw["grid"] = g
        if name == "lattice_scale_u32":
            kw["deposit_mode"] = _abi.P3M_DEPOSIT_U32
        return scenarios.lattice_scale(**kw)
    if name == "batch":
        return scenarios.batch(**({"sims": sims} if sims else {}))
    if name == "adjoint":
        kw = {}
        if bodies:
            kw["n_cluster"] = bodies - 1000
        if g:
            kw["grid"] = g
        return scenarios.adjoint_cluster(**kw)
    raise SystemExit(f"unknown workload {name}")


def run_only(args) -> None:
    """The workload's initial pass and --steps steps, nothing timed or
    printed but a final 'ok': the target of the committed Nsight Compute
    captures (adjoint: a checkpointed rollout of --steps steps and its
    backward pass; batch: --steps batch steps)."""
    import torch

    torch.cuda.set_device(0)
    if args.workload == "batch":
        from gravity_b200.batch import GravityBatch

        scs = make_workload("batch", sims=args.sims)
        with GravityBatch([sc.config for sc in scs]) as b:
            if args.batch_form == "persistent":
                b.set_persistent(True)
            elif args.batch_form == "per_stage":
                b.set_persistent(False)
            elif args.batch_form == "per_simulation":
                b.set_fused(False)
            for i, sc in enumerate(scs):
                b.upload(i, sc.bodies, sc.materials)
            b.initialize_acceleration()
            b.step(args.steps)
            b.synchronize()
        print("ok", sum(sc.n for sc in scs))
        return
    from gravity_b200.pipeline import GravityPipeline

    sc = make_workload(args.workload, args.bodies, args.grid)
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        if args.workload == "adjoint":
            from gravity_b200.adjoint import Rollout

            r = Rollout(p, sc.n, args.steps, checkpoint_interval=max(1, args.steps // 2))
            r.forward()
            seed = np.zeros((sc.n, 4), np.float32)
            seed[-1000:, 0] = 1.0
            r.backward(seed)
        else:
            p.initialize_acceleration(sc.n)
            p.step(sc.n, args.steps)
            if args.previews:
                # A fan of aim previews on the field of the last step.
                w_px, h_px = sc.config.viewport_width, sc.config.viewport_height
                ang = np.linspace(0.0, 2.0 * np.pi, args.previews, endpoint=False)
                o = np.tile(np.array([0.3 * w_px, 0.5 * h_px], np.float32), (args.previews, 1))
                v = (300.0 * np.stack([np.cos(ang), np.sin(ang)], axis=1)).astype(np.float32)
                p.trajectories(sc.n, o, v, steps=1024)
        p.synchronize()
    print("ok", sc.n)


def mesh_sizes(sc):
    g = sc.config.gravity
    P = g.grid_width * g.grid_height
    k = 4 if sc.config.bounded else 1
    return P, P * k


def stage_bytes(sc, stage: str, radix_passes: int) -> float:
    """Algorithmic bytes of one launch of a stage: the compulsory traffic of
    its inputs and outputs for N bodies, P physical cells, M mesh cells and
    p radix passes (body records 16 B, accelerations 8 B, cell tables 4 B per
    word, mesh words 4 or 8 B)."""
    n = sc.n
    P, M = mesh_sizes(sc)
    i64 = sc.config.deposit_mode == 1
    d = 8 if i64 else 4
    if stage == "drift":
        return 48.0 * n
    if stage == "cell_lists":
        return 16.0 * radix_passes * n + 44.0 * n + 12.0 * P
    if stage == "deposit":
        return 16.0 * n + 2.0 * d * M
    if stage == "forward_fft":
        return (d + 4.0) * M
    if stage == "spectral":
        return 16.0 * M
    if stage == "inverse_fft":
        return 16.0 * M
    if stage == "kick":
        return 48.0 * n + 8.0 * P
    if stage == "short_range":
        return 24.0 * n + 12.0 * P
    if stage == "spatial_sort":
        return 16.0 * radix_passes * n + 88.0 * n
    return 0.0


def radix_passes_for_bits(bits: int) -> int:
    """Passes of the library's radix sort over `bits` key bits: 8-bit digits,
    or 9-bit digits where they save a pass."""
    p = (bits + 7) // 8
    if p > 1 and (bits + 8) // 9 < p:
        p = (bits + 8) // 9
    return p


def radix_passes_for(count: int) -> int:
    return radix_passes_for_bits(max(1, (count - 1).bit_length()))


def read_traffic(stage: str, workload: str):
    """DRAM bytes per launch from a committed ncu summary, if one exists
    (a line `traffic_bytes_per_launch: <int>` in profiles/<stage>_<workload>*.md)."""
    for f in sorted((REPO / "profiles").glob(f"{stage}_{workload}*.md")):
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", f.read_text())
        if m:
            return float(m.group(1))
    return None


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# -------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-i", str(self.device_index), "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
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
        self._t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# -------------------------------------------------------------- CPU baseline
def short_range_xu(sc, ms_per_launch: float, clk) -> dict | None:
    """The exp2/reciprocal floor of the two-slot short range: per body and
    non-home stencil cell two exp2 and two reciprocals (one pair term per
    slot), on the MUFU unit's 16 results per clock per SM. The home cell's
    walk adds a few more, so the floor is a lower bound. None for the list
    form (the exact limit is not 2, or under one body per two cells)."""
    import torch
    from gravity_b200.config import neighbor_radii

    g = sc.config.gravity
    cells = g.grid_width * g.grid_height
    if g.exact_neighbor_body_limit != 2 or 2 * sc.n < cells or not ms_per_launch:
        return None
    rx, ry = neighbor_radii(sc.config)
    ops = 4 * ((2 * rx + 1) * (2 * ry + 1) - 1) * sc.n
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz")
    if not mhz:
        return None
    floor_ms = ops / (16.0 * sms * mhz * 1e6) * 1e3
    return {"unit": "MUFU ops (ex2, rcp)", "ops_per_launch": ops, "per_sm_clock": 16,
            "sms": sms, "sm_mhz": mhz, "floor_ms": floor_ms, "frac": floor_ms / ms_per_launch}


def cpu_oracle_rate(sc, budget_s: float, threads: int | None = None, warmup: int = 1,
                    max_steps: int | None = None):
    """bodies*steps/s of the CPU oracle on this workload: initialisation and
    `warmup` steps untimed, then steps until `budget_s` is spent."""
    import oracle

    if threads:
        oracle.set_threads(threads)
    used = oracle.max_threads()
    sim = oracle.OracleSim(sc.config)
    sim.upload(sc.bodies, sc.materials)
    sim.initialize_acceleration(sc.n)
    for _ in range(warmup):
        sim.step(sc.n)
    steps = 0
    t0 = time.perf_counter()
    while True:
        sim.step(sc.n)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_steps and steps >= max_steps):
            break
    sim.close()
    return sc.n * steps / el, steps, el, used


# ------------------------------------------------------------------ helpers
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws: int, local: int):
    """One process per GPU over NCCL (barrier and max-over-ranks timing only:
    the replicas exchange no data). Without CUDA (the CPU tests) the same
    calls run over gloo."""
    import torch
    import torch.distributed as dist

    if ws > 1:
        from datetime import timedelta
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=timedelta(seconds=120))
    return dist if ws > 1 else None


def allreduce_max(dist, value: float) -> float:
    if dist is None:
        return value
    import torch

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def force_error_vs_fp64(pipe, sc) -> float:
    """Relative RMS error of the P3M accelerations of a seeded 4096-body
    subsample against the FP64 direct sum, on the initial state."""
    n = sc.n
    rng = np.random.default_rng(4096)
    targets = np.sort(rng.choice(n, size=min(FORCE_SAMPLE, n), replace=False)).astype(np.int32)
    pipe.upload(sc.bodies, sc.materials)
    pipe.initialize_acceleration(n)
    a = pipe.acceleration(n)[targets].astype(np.float64)
    ref = pipe.direct_accel_f64(n, targets)
    return float(np.sqrt(np.sum((a - ref) ** 2) / np.sum(ref ** 2)))


# -------------------------------------------------------------------- arms
def run_reference(args, ws, rank):
    if rank != 0:
        return
    if args.workload == "batch":
        scs = make_workload("batch")
        budget = max(5.0, min(90.0, float(args.steps) * 2.0))
        rate, sims, el, used = cpu_oracle_batch_rate(scs, budget, threads=os.cpu_count())
        sample = (f"the first {sims} of {len(scs)} simulations, 4 P3M steps each ({el:.1f} s) "
                  f"after initialisation and 1 untimed step")
        line = {
            "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": ws,
            "steps": 4, "warmup": 1, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": batch_config(scs, args),
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": used, "kind": "port",
                             "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    sc = make_workload(args.workload, args.bodies, args.grid)
    threads = os.cpu_count() or 1
    budget = max(5.0, min(90.0, float(args.steps) * 2.0))
    rate, steps, el, used = cpu_oracle_rate(sc, budget, threads=threads,
                                            warmup=args.warmup, max_steps=args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": ws,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 * el / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": workload_config(sc, args),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": used, "kind": "port",
                         "sample": f"{steps} P3M steps of the {sc.n}-body {args.workload} "
                                   f"workload ({el:.1f} s) after initialisation and "
                                   f"{args.warmup} untimed step(s)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batch_config(scs, args):
    from collections import Counter

    grids = Counter(f"{sc.config.gravity.grid_width}x{sc.config.gravity.grid_height}" for sc in scs)
    ns = [sc.n for sc in scs]
    return {
        "workload": "batch", "simulations": len(scs), "n_bodies": int(sum(ns)),
        "n_min": int(min(ns)), "n_max": int(max(ns)), "grids": dict(sorted(grids.items())),
        "boundary": "torus", "deposit": "uint32", "px_per_cell": 5,
        "dt": scs[0].config.time_step, "drift_substeps": scs[0].config.drift_substeps,
        "spatial_sort_interval": scs[0].config.spatial_sort_interval,
        "l2": "flushed (256 MiB write) before every timed step",
        "parallelism": "replicas" if args.gpus > 1 else "single",
    }


def cpu_oracle_batch_rate(scs, budget_s: float, threads: int | None = None):
    """bodies*steps/s of the CPU oracle over the batch's simulations taken in
    order, each initialised and stepped once untimed, then stepped 4 times
    timed, until `budget_s` of timed work is spent."""
    import oracle

    if threads:
        oracle.set_threads(threads)
    used = oracle.max_threads()
    work = 0
    el = 0.0
    sims = 0
    for sc in scs:
        sim = oracle.OracleSim(sc.config)
        sim.upload(sc.bodies, sc.materials)
        sim.initialize_acceleration(sc.n)
        sim.step(sc.n)
        t0 = time.perf_counter()
        for _ in range(4):
            sim.step(sc.n)
        el += time.perf_counter() - t0
        sim.close()
        work += 4 * sc.n
        sims += 1
        if el >= budget_s:
            break
    return work / el, sims, el, used


def workload_config(sc, args, name=None):
    g = sc.config.gravity
    P, M = mesh_sizes(sc)
    mw = g.grid_width * (2 if sc.config.bounded else 1)
    mh = g.grid_height * (2 if sc.config.bounded else 1)
    return {
        "workload": name or args.workload, "n_bodies": sc.n,
        "grid": f"{g.grid_width}x{g.grid_height}", "fft_mesh": f"{mw}x{mh}",
        "boundary": "walls" if sc.config.bounded else "torus",
        "deposit": "int64" if sc.config.deposit_mode == 1 else "uint32",
        "viewport_px": f"{sc.config.viewport_width}x{sc.config.viewport_height}",
        "dt": sc.config.time_step, "drift_substeps": sc.config.drift_substeps,
        "spatial_sort_interval": sc.config.spatial_sort_interval,
        "l2": "flushed (256 MiB write) before every timed step",
        "parallelism": "replicas" if args.gpus > 1 else "single",
    }


def measure_steps(pipe, sc, args, stream, flush, dist, local, steps, warmup, sample_clocks):
    """The autotuner picks the launch shapes (the state is put back), then
    device-timed steps (graphs replayed, state resident in HBM, L2 flushed
    before each step), then the same steps again from the initial state with
    stage events, then the e2e pass through the public API with page-locked
    host buffers."""
    import torch

    from gravity_b200.pipeline import PinnedArray, kernel_launches

    ws = dist.get_world_size() if dist else 1
    n = sc.n
    pipe.upload(sc.bodies, sc.materials)
    pipe.initialize_acceleration(n)
    tuned = pipe.autotune(n, 3)
    for _ in range(warmup):
        pipe.step(n)
    pipe.synchronize()
    if dist:
        dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    clocks = ClockSampler(local) if sample_clocks else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    launches0 = kernel_launches()
    with torch.cuda.stream(stream):
        for i in range(steps):
            flush.zero_()
            starts[i].record(stream)
            pipe.step(n)
            stops[i].record(stream)
    torch.cuda.synchronize()
    pipe.synchronize()
    launches = kernel_launches() - launches0
    clk = clocks.stop() if clocks else None
    total_ms = sum(a.elapsed_time(b) for a, b in zip(starts, stops))
    total_ms = allreduce_max(dist, total_ms)
    if dist:
        dist.barrier()
    value = ws * n * steps / (total_ms / 1000.0)

    # ---- per-stage device time: the same steps from the same initial state
    # (the bodies cluster as they evolve, which changes the stages' work),
    # with stage events recorded (kernels launched one by one; the value pass
    # above replays graphs).
    pipe.upload(sc.bodies, sc.materials)
    pipe.initialize_acceleration(n)
    for _ in range(warmup):
        pipe.step(n)
    pipe.profile_enable(True)
    with torch.cuda.stream(stream):
        for i in range(steps):
            flush.zero_()
            pipe.step(n)
    stages = pipe.profile_read()
    pipe.profile_enable(False)

    # ---- e2e: through the public API with page-locked host buffers
    e2e_steps = steps if args.e2e_steps is None else min(steps, args.e2e_steps)
    hb = PinnedArray((n, 4))
    hm = PinnedArray((n, 4))
    out = PinnedArray((n, 4))
    hb.array[:] = sc.bodies
    hm.array[:] = sc.materials
    pipe.upload_n(n, hb.array, hm.array)
    pipe.initialize_acceleration(n)
    # The host then holds the state as the library keeps it after the
    # warm-up (bodies and materials in the order of the last reorder), as a
    # host that reads the state back every step does, and uploads that.
    for _ in range(max(warmup, 2)):
        pipe.step(n)
    pipe.download_into(n, hb.array, hm.array)
    pipe.upload_n(n, hb.array, hm.array)
    for _ in range(min(warmup, 3)):
        pipe.upload_n(n, hb.array)
        pipe.step(n)
        pipe.download_into(n, out.array)
    if dist:
        dist.barrier()
    # Serial: upload, step, download, each call returning when its copy is
    # done (L2 flushed before each step, outside its time).
    e2e_s = 0.0
    for _ in range(e2e_steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        pipe.synchronize()
        t0 = time.perf_counter()
        pipe.upload_n(n, hb.array)
        pipe.step(n)
        pipe.download_into(n, out.array)
        e2e_s += time.perf_counter() - t0
    e2e_s = allreduce_max(dist, e2e_s)
    e2e_serial = ws * n * e2e_steps / e2e_s
    # Pipelined (p3m_step_io): every step uploads its input and downloads its
    # result as above, but the upload of step k+1 and the download of step k
    # run on the copy engines while the steps compute. The whole run, L2
    # flushes included, is timed, up to the last download.
    for _ in range(min(warmup, 3)):
        pipe.step_io(n, hb.array, out.array)
    pipe.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        pipe.step_io(n, hb.array, out.array)
    pipe.synchronize()
    e2e_pipe_s = allreduce_max(dist, time.perf_counter() - t0)
    e2e_value = ws * n * e2e_steps / e2e_pipe_s
    for a in (hb, hm, out):
        a.free()
    # No bounded device wait may have given up during any of it.
    timeouts = pipe.wait_timeouts()
    if timeouts:
        raise SystemExit(f"{timeouts} look-back wait(s) of the sort gave up: results invalid")
    return {"value": value, "ms_per_step": total_ms / steps, "stages": stages,
            "launches": launches, "clocks": clk,
            "autotuned": {"fft_lines_per_cta": tuned[0] or "auto", "short_range_threads": tuned[1]},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 16 * n,
                    "d2h_bytes_per_step": 16 * n, "steps": e2e_steps,
                    "mode": "pipelined: p3m_step_io, copies overlapped with the steps",
                    "serial_value": e2e_serial}}


def stage_table(sc, stages):
    """Per-stage average launch time and achieved algorithmic GB/s."""
    from gravity_b200.config import sort_axis_bits

    P, M = mesh_sizes(sc)
    cell_passes = radix_passes_for(P)
    morton_bits = sort_axis_bits(sc.config.viewport_width) + sort_axis_bits(sc.config.viewport_height)
    morton_passes = radix_passes_for_bits(morton_bits)
    peak, _ = measured_peaks()
    rows = {}
    for name, (ms, cnt) in stages.items():
        if cnt == 0:
            continue
        passes = morton_passes if name == "spatial_sort" else cell_passes
        avg_ms = ms / cnt
        b = stage_bytes(sc, name, passes)
        gbs = b / (avg_ms / 1000.0) / 1e9 if avg_ms > 0 else None
        rows[name] = {"ms_per_launch": avg_ms, "launches": cnt, "algorithmic_bytes": b,
                      "gbs": gbs, "frac_of_measured_hbm": gbs / peak if gbs else None}
    return rows


def force_errors_by_form(sc, pipe_err):
    """RMS force error against the FP64 direct sum on the same seeded
    4096-body subsample (initial state) for this line's deposit form, the
    other deposit form on the GPU, and the oracle's FP32 path (the
    reference's uint32 deposit)."""
    import oracle
    from gravity_b200 import _abi
    from gravity_b200.pipeline import GravityPipeline

    n = sc.n
    rng = np.random.default_rng(4096)
    targets = np.sort(rng.choice(n, size=min(FORCE_SAMPLE, n), replace=False)).astype(np.int32)
    other_mode = _abi.P3M_DEPOSIT_U32 if sc.config.deposit_mode == _abi.P3M_DEPOSIT_I64 else _abi.P3M_DEPOSIT_I64
    names = {_abi.P3M_DEPOSIT_U32: "uint32", _abi.P3M_DEPOSIT_I64: "int64"}
    out = {names[sc.config.deposit_mode]: pipe_err}
    with GravityPipeline(sc.config.with_(deposit_mode=other_mode)) as other:
        other.upload(sc.bodies, sc.materials)
        other.initialize_acceleration(n)
        a = other.acceleration(n)[targets].astype(np.float64)
        ref = other.direct_accel_f64(n, targets)
    out[names[other_mode]] = float(np.sqrt(np.sum((a - ref) ** 2) / np.sum(ref ** 2)))
    ocfg = sc.config.with_(deposit_mode=_abi.P3M_DEPOSIT_U32)
    with oracle.OracleSim(ocfg) as sim:
        sim.upload(sc.bodies, sc.materials)
        sim.initialize_acceleration(n)
        a = sim.download(n)[2][targets].astype(np.float64)
    out["oracle_fp32_uint32"] = float(np.sqrt(np.sum((a - ref) ** 2) / np.sum(ref ** 2)))
    return out


def run_b200(args, ws, rank, local):
    import torch

    from gravity_b200.pipeline import GravityPipeline

    dist = init_dist(ws, local)
    torch.cuda.set_device(local)
    sc = make_workload(args.workload, args.bodies, args.grid)
    n = sc.n
    pipe = GravityPipeline(sc.config)
    stream = torch.cuda.ExternalStream(pipe.stream_handle())
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    force_err = force_error_vs_fp64(pipe, sc) if rank == 0 else None
    m = measure_steps(pipe, sc, args, stream, flush, dist, local, args.steps, args.warmup, True)
    value, ms_per_step, stages, launches, clk = (m["value"], m["ms_per_step"], m["stages"],
                                                 m["launches"], m["clocks"])

    # ---- aim previews on the field of the last step (S/trajectory.comp):
    # one preview, then a fan of 256, 1024 steps each (host wall clock,
    # synchronous calls, vertices copied back).
    previews = None
    if rank == 0 and sc.config.mutual_gravity:
        w_px, h_px = sc.config.viewport_width, sc.config.viewport_height
        ang = np.linspace(0.0, 2.0 * np.pi, 256, endpoint=False)
        fan_o = np.tile(np.array([0.3 * w_px, 0.5 * h_px], np.float32), (256, 1))
        fan_v = (300.0 * np.stack([np.cos(ang), np.sin(ang)], axis=1)).astype(np.float32)
        pipe.trajectories(n, fan_o, fan_v, steps=1024)  # buffers sized, code warm
        t0 = time.perf_counter()
        pipe.trajectories(n, fan_o[:1], fan_v[:1], steps=1024)
        one = time.perf_counter() - t0
        t0 = time.perf_counter()
        pipe.trajectories(n, fan_o, fan_v, steps=1024)
        many = time.perf_counter() - t0
        previews = {"steps": 1024, "single_ms": 1000.0 * one, "fan": 256,
                    "fan_ms": 1000.0 * many, "preview_steps_per_s": 256 * 1024 / many}
    pipe.close()

    # ---- the plain configuration beside it: 400,000 Plummer bodies inside
    # walls with the reference's uint32 deposit (a shorter run).
    plain = None
    if args.workload == "lattice_scale" and not args.no_plain:
        psc = make_workload("plummer_walls")
        ppipe = GravityPipeline(psc.config)
        pstream = torch.cuda.ExternalStream(ppipe.stream_handle())
        perr = force_error_vs_fp64(ppipe, psc) if rank == 0 else None
        psteps = min(args.steps, 200)
        pm = measure_steps(ppipe, psc, args, pstream, flush, dist, local, psteps,
                           args.warmup, False)
        ppipe.close()
        if rank == 0:
            prow = stage_table(psc, pm["stages"])
            plain = {"workload": "plummer_walls", "config": workload_config(psc, args, "plummer_walls"),
                     "value": pm["value"], "ms_per_step": pm["ms_per_step"], "steps": psteps,
                     "e2e": pm["e2e"], "force_rms_err_vs_fp64": perr, "stages": prow,
                     "short_range_xu": short_range_xu(
                         psc, prow.get("short_range", {}).get("ms_per_launch"), clk),
                     "autotuned": pm["autotuned"], "gpu_launches": pm["launches"]}

    if rank == 0:
        peak, peak_kind = measured_peaks()
        stage_rows = stage_table(sc, stages)
        dominant = max(stage_rows, key=lambda k: stage_rows[k]["ms_per_launch"] * stage_rows[k]["launches"])
        dom = stage_rows[dominant]
        achieved = dom["gbs"]
        traffic = read_traffic(dominant, args.workload)
        errors = force_errors_by_form(sc, force_err) if not args.no_form_errors else None
        cpu = None
        if not args.no_cpu_baseline:
            rate, steps, el, used = cpu_oracle_rate(sc, args.cpu_seconds, threads=os.cpu_count())
            rate1, steps1, el1, _ = cpu_oracle_rate(sc, min(args.cpu_seconds, 10.0), threads=1,
                                                    max_steps=steps)
            cpu = {"value": rate, "unit": UNIT, "cores": used, "kind": "port",
                   "sample": f"{steps} P3M steps of the {n}-body {args.workload} workload "
                             f"({el:.1f} s) after initialisation and 1 untimed step",
                   "value_1_thread": rate1,
                   "sample_1_thread": f"{steps1} steps ({el1:.1f} s) on one thread"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(sc, args),
            "force_rms_err_vs_fp64": force_err,
            "force_rms_err_vs_fp64_by_form": errors,
            "autotuned": m["autotuned"],
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak if achieved else None,
                         "traffic": traffic, "peak_source": peak_kind,
                         "xu": short_range_xu(sc, dom["ms_per_launch"], clk)
                         if dominant == "short_range" else None},
            "roofline_hbm_stages": {k: stage_rows[k]["frac_of_measured_hbm"]
                                    for k in ("deposit", "kick") if k in stage_rows},
            "stages": stage_rows,
            "cpu_baseline": cpu,
            "e2e": m["e2e"],
            "gpu_launches": launches,
            "clocks": clk,
            "previews": previews,
            "plain_form": plain,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args, ws, rank, local):
    """256 simulations of uneven sizes stepped together (one graph launch per
    batch step), after the autotuner has picked the form -- one launch per
    stage or one persistent kernel launch -- and the launch shapes by timing
    whole batch steps. The other form, and the simulations as serial runs,
    are timed beside it."""
    import torch

    from gravity_b200.batch import GravityBatch
    from gravity_b200.pipeline import GravityPipeline, PinnedArray, kernel_launches

    dist = init_dist(ws, local)
    torch.cuda.set_device(local)
    scs = make_workload("batch")
    total_n = sum(sc.n for sc in scs)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    batch = GravityBatch([sc.config for sc in scs])
    stream = torch.cuda.ExternalStream(batch.stream_handle())

    def reset():
        for i, sc in enumerate(scs):
            batch.upload(i, sc.bodies, sc.materials)
        batch.initialize_acceleration()

    reset()
    batch.step(2)
    tuned = batch.autotune(trial_steps=3)
    reset()
    # Every captured graph (body counts x reorder phase x buffers) is built
    # during the warm-up.
    warmup = max(args.warmup, 4)
    batch.step(warmup)
    batch.synchronize()
    if dist:
        dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = kernel_launches()
    with torch.cuda.stream(stream):
        for i in range(args.steps):
            flush.zero_()
            starts[i].record(stream)
            batch.step(1)
            stops[i].record(stream)
    torch.cuda.synchronize()
    batch.synchronize()
    launches = kernel_launches() - launches0
    clk = clocks.stop()
    total_ms = allreduce_max(dist, sum(a.elapsed_time(b) for a, b in zip(starts, stops)))
    value = ws * total_n * args.steps / (total_ms / 1000.0)
    plan = batch.plan_info()
    chosen_persistent = plan["persistent"]
    if chosen_persistent:
        plan["phase_ms_last_step"] = [round(t, 5) for t in batch.phase_times()]
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    per_sm = plan["ctas"] // sms if plan["ctas"] else 0

    # ---- the same batch in the other form (persistent <-> one launch per
    # stage), timed the same way.
    batch.set_persistent(not chosen_persistent, per_sm)
    batch.step(warmup)
    batch.synchronize()
    with torch.cuda.stream(stream):
        for i in range(args.steps):
            flush.zero_()
            starts[i].record(stream)
            batch.step(1)
            stops[i].record(stream)
    torch.cuda.synchronize()
    batch.synchronize()
    other = batch.plan_info()
    other_ms = allreduce_max(dist, sum(a.elapsed_time(b) for a, b in zip(starts, stops)))
    other["value"] = ws * total_n * args.steps / (other_ms / 1000.0)
    other["ms_per_step"] = other_ms / args.steps
    if other["persistent"]:
        other["phase_ms_last_step"] = [round(t, 5) for t in batch.phase_times()]
    plan["other_form"] = other
    batch.set_persistent(chosen_persistent, per_sm)
    batch.step(warmup)
    batch.synchronize()

    # ---- e2e: every step uploads every simulation's body state from
    # page-locked memory (materials once, before timing), steps the batch and
    # reads every simulation's bodies back.
    e2e_steps = args.steps if args.e2e_steps is None else min(args.steps, args.e2e_steps)
    hb = [PinnedArray((sc.n, 4)) for sc in scs]
    hm = [PinnedArray((sc.n, 4)) for sc in scs]
    out = [PinnedArray((sc.n, 4)) for sc in scs]
    views = []
    # The state as the batch keeps it after the runs above (bodies and
    # materials in the order of the last reorder), as a host that reads the
    # state back every step holds it; that is what every step uploads.
    for i, sc in enumerate(scs):
        views.append(batch.simulation(i))
        views[i].download_into(sc.n, hb[i].array, hm[i].array)
        batch.upload(i, hb[i].array, hm[i].array)
    e2e_s = 0.0
    for it in range(min(args.warmup, 3) + e2e_steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        batch.synchronize()
        t0 = time.perf_counter()
        for i in range(len(scs)):
            batch.upload(i, hb[i].array)
        batch.step(1)
        batch.synchronize()
        for i, sc in enumerate(scs):
            views[i].download_into(sc.n, out[i].array)
        if it >= min(args.warmup, 3):
            e2e_s += time.perf_counter() - t0
    e2e_s = allreduce_max(dist, e2e_s)
    e2e_serial = ws * total_n * e2e_steps / e2e_s
    # Pipelined (p3m_batch_step_io): all simulations' bodies back to back in
    # one page-locked array per direction, one copy each way per step,
    # overlapping the neighbouring steps; the whole run is timed.
    cat_in = PinnedArray((total_n, 4))
    cat_out = PinnedArray((total_n, 4))
    cat_in.array[:] = np.concatenate([h.array for h in hb])
    for _ in range(min(args.warmup, 3) + 1):
        batch.step_io(cat_in.array, cat_out.array)
    batch.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        batch.step_io(cat_in.array, cat_out.array)
    batch.synchronize()
    e2e_pipe_s = allreduce_max(dist, time.perf_counter() - t0)
    e2e_value = ws * total_n * e2e_steps / e2e_pipe_s
    cat_in.free()
    cat_out.free()

    # ---- per-stage device time: every simulation stepped on its own with
    # stage events (no graphs), summed over simulations.
    stage_rows = {}
    for i, sc in enumerate(scs):
        views[i].profile_enable(True)
        for _ in range(2):
            views[i].step(sc.n)
        prof = views[i].profile_read()
        views[i].profile_enable(False)
        P, M = mesh_sizes(sc)
        for name, (ms, cnt) in prof.items():
            if cnt == 0:
                continue
            passes = radix_passes_for(P)
            if name == "spatial_sort":
                from gravity_b200.config import sort_axis_bits
                passes = radix_passes_for_bits(sort_axis_bits(sc.config.viewport_width)
                                               + sort_axis_bits(sc.config.viewport_height))
            r = stage_rows.setdefault(name, {"ms": 0.0, "launches": 0, "bytes": 0.0})
            r["ms"] += ms
            r["launches"] += cnt
            r["bytes"] += stage_bytes(sc, name, passes) * cnt
    for v in views:
        v.close()
    batch.close()

    # ---- the same simulations as serial runs of the plain path: one context
    # each, run alone for its steps (graph-replayed) before the next starts
    pipes = []
    for sc in scs:
        p = GravityPipeline(sc.config)
        p.upload(sc.bodies, sc.materials)
        p.initialize_acceleration(sc.n)
        pipes.append(p)
    for _ in range(warmup):
        for p, sc in zip(pipes, scs):
            p.step(sc.n)
    for p in pipes:
        p.synchronize()
    indiv_steps = min(args.steps, 30)
    t0 = time.perf_counter()
    for p, sc in zip(pipes, scs):
        p.step(sc.n, indiv_steps)
        p.synchronize()
    serial_value = total_n * indiv_steps / (time.perf_counter() - t0)
    # ... and all contexts stepped in turn from the host without waiting
    # (their streams overlap on the GPU).
    t0 = time.perf_counter()
    for _ in range(indiv_steps):
        for p, sc in zip(pipes, scs):
            p.step(sc.n)
    for p in pipes:
        p.synchronize()
    overlapped_value = total_n * indiv_steps / (time.perf_counter() - t0)
    for p in pipes:
        p.close()
    for a in hb + hm + out:
        a.free()

    if rank == 0:
        peak, peak_kind = measured_peaks()
        rows = {k: {"ms_per_launch": v["ms"] / v["launches"], "launches": v["launches"],
                    "algorithmic_bytes": v["bytes"] / v["launches"],
                    "gbs": v["bytes"] / (v["ms"] / 1000.0) / 1e9 if v["ms"] > 0 else None}
                for k, v in stage_rows.items()}
        dominant = max(rows, key=lambda k: stage_rows[k]["ms"])
        achieved = rows[dominant]["gbs"]
        cpu = None
        if not args.no_cpu_baseline:
            rate, sims, el, used = cpu_oracle_batch_rate(scs, args.cpu_seconds, threads=os.cpu_count())
            cpu = {"value": rate, "unit": UNIT, "cores": used, "kind": "port",
                   "sample": f"the first {sims} of {len(scs)} simulations, 4 P3M steps each "
                             f"({el:.1f} s) after initialisation and 1 untimed step"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": batch_config(scs, args),
            "autotuned": [{"grid": f"{r[0]}x{r[1]}", "fft_lines_per_cta": r[2] or "auto",
                           "short_range_threads": r[3]} for r in tuned],
            "plan": plan,
            "serial_runs_value": serial_value,
            "overlapped_contexts_value": overlapped_value,
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak if achieved else None,
                         "traffic": None, "peak_source": peak_kind,
                         "note": "stage bytes and device time summed over the simulations"},
            "stages": rows,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 16 * total_n,
                    "d2h_bytes_per_step": 16 * total_n, "steps": e2e_steps,
                    "mode": "pipelined: p3m_batch_step_io, copies overlapped with the steps",
                    "serial_value": e2e_serial},
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


ADJOINT_GROUP = slice(99_000, 100_000)   # the projectile disc
ADJOINT_V0_PX = (-60.0, 45.0)             # launch velocity, px/s
ADJOINT_TARGET_PX = (1900.0, 760.0)       # target of the disc's centroid, px
ADJOINT_INTERVAL = 16
ADJOINT_FD_H = 1e-2                       # px/s


def run_adjoint(args, ws, rank, local):
    """Forward (checkpointed) + backward of the T-step rollout; value =
    differentiated bodies*steps/s. Also the plain forward's rate, the
    backward/forward cost ratio, the launch-velocity gradient against central
    differences, and (with --fp64-check) against the FP64 reference."""
    import torch

    from gravity_b200.adjoint import Rollout, launch_velocity_objective
    from gravity_b200.pipeline import GravityPipeline, PinnedArray, kernel_launches

    dist = init_dist(ws, local)
    torch.cuda.set_device(local)
    sc = make_workload("adjoint")
    n, T = sc.n, sc.steps
    group = np.arange(n)[ADJOINT_GROUP]
    base = sc.bodies.copy()
    base[group, 2] = ADJOINT_V0_PX[0] / sc.config.viewport_width
    base[group, 3] = ADJOINT_V0_PX[1] / sc.config.viewport_height
    pipe = GravityPipeline(sc.config)
    pipe.upload(base, sc.materials)
    stream = torch.cuda.ExternalStream(pipe.stream_handle())
    roll = Rollout(pipe, n, T, checkpoint_interval=ADJOINT_INTERVAL)
    x0 = torch.tensor(base, device="cuda")
    seed = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    seed[group, 0] = 1.0
    grad = torch.empty_like(seed)
    final = torch.empty_like(seed)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def plain_forward():
        pipe.initialize_acceleration(n)
        pipe.step(n, T)

    # ---- plain forward: initializeAcceleration + T steps, device-timed
    for _ in range(args.warmup):
        pipe.upload(base)
        plain_forward()
    pipe.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    fwd_ms = []
    for _ in range(max(3, min(args.steps, 10))):
        pipe.upload(base)
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[0].record(stream)
        plain_forward()
        with torch.cuda.stream(stream):
            ev[1].record(stream)
        torch.cuda.synchronize()
        fwd_ms.append(ev[0].elapsed_time(ev[1]))
    plain_ms = statistics.median(fwd_ms)

    # ---- value: forward with checkpoints + backward, device-resident
    for _ in range(args.warmup):
        roll.forward(x0, final)
        roll.backward(seed, out=grad)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = kernel_launches()
    f_ms, b_ms = [], []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[0].record(stream)
        roll.forward(x0, final)
        with torch.cuda.stream(stream):
            ev[1].record(stream)
        roll.backward(seed, out=grad)
        with torch.cuda.stream(stream):
            ev[2].record(stream)
        torch.cuda.synchronize()
        f_ms.append(ev[0].elapsed_time(ev[1]))
        b_ms.append(ev[1].elapsed_time(ev[2]))
    launches = kernel_launches() - launches0
    clk = clocks.stop()
    total_ms = allreduce_max(dist, sum(f_ms) + sum(b_ms))
    value = ws * n * T * args.steps / (total_ms / 1000.0)

    # ---- e2e: host initial state in, host gradient out
    hb = PinnedArray((n, 4))
    hs = PinnedArray((n, 4))
    hg = PinnedArray((n, 4))
    hf = PinnedArray((n, 4))
    hb.array[:] = base
    hs.array[:] = seed.cpu().numpy()
    e2e_steps = max(1, min(args.steps, args.e2e_steps or args.steps))
    e2e_s = 0.0
    for it in range(1 + e2e_steps):
        t0 = time.perf_counter()
        roll.forward(hb.array, hf.array)
        roll.backward(hs.array, out=hg.array)
        if it > 0:
            e2e_s += time.perf_counter() - t0
    e2e_s = allreduce_max(dist, e2e_s)
    e2e_value = ws * n * T * e2e_steps / e2e_s

    # ---- gradient checks on the launch velocity
    v0 = np.array(ADJOINT_V0_PX)
    obj = launch_velocity_objective(roll, sc.bodies, group, v0, ADJOINT_TARGET_PX)
    def central(h):
        out = []
        for k in range(2):
            e = np.zeros(2)
            e[k] = h
            lp = launch_velocity_objective(roll, sc.bodies, group, v0 + e, ADJOINT_TARGET_PX, False).loss
            lm = launch_velocity_objective(roll, sc.bodies, group, v0 - e, ADJOINT_TARGET_PX, False).loss
            out.append((lp - lm) / (2 * h))
        return np.array(out)

    fd = central(ADJOINT_FD_H)
    fd_err = float(np.linalg.norm(obj.grad_velocity_px - fd) / np.linalg.norm(fd))
    # The quotient at neighbouring steps: where they disagree with each
    # other the loss is not smooth at that scale.
    fd_spread = {str(h): central(h).tolist() for h in (1e-1, 1e-3)}
    fp64 = None
    if args.fp64_check and rank == 0:
        import oracle

        ref = oracle.Adjoint64(sc.config, sc.materials)
        b = sc.bodies.astype(np.float64)
        b[group, 2] = v0[0] / sc.config.viewport_width
        b[group, 3] = v0[1] / sc.config.viewport_height
        t0 = time.perf_counter()
        fin, _ = ref.forward(b, T)
        scale = np.array([sc.config.viewport_width, sc.config.viewport_height], np.float64)
        d = fin[group, :2] - b[group, :2]
        d -= np.round(d)
        c = (b[group, :2] + d).mean(axis=0) * scale
        s64 = np.zeros((n, 4))
        s64[group, 0] = 2 * (c[0] - ADJOINT_TARGET_PX[0]) * scale[0] / len(group)
        s64[group, 1] = 2 * (c[1] - ADJOINT_TARGET_PX[1]) * scale[1] / len(group)
        g64, _ = ref.backward(s64)
        gv64 = np.array([g64[group, 2].sum() / scale[0], g64[group, 3].sum() / scale[1]])
        g = obj.grad_bodies.astype(np.float64)
        fp64 = {"launch_velocity_rel_err": float(np.linalg.norm(obj.grad_velocity_px - gv64) / np.linalg.norm(gv64)),
                "all_bodies_rel_err": float(np.linalg.norm(g - g64) / np.linalg.norm(g64)),
                "grad_velocity_px_fp64": gv64.tolist(), "host_seconds": time.perf_counter() - t0}
    for a in (hb, hs, hg, hf):
        a.free()

    if rank == 0:
        peak, peak_kind = measured_peaks()
        f_avg, b_avg = statistics.mean(f_ms), statistics.mean(b_ms)
        cpu = None
        if not args.no_cpu_baseline:
            rate, steps, el, used = cpu_oracle_rate(sc, args.cpu_seconds, threads=os.cpu_count())
            cpu = {"value": rate, "unit": UNIT, "cores": used, "kind": "port",
                   "sample": f"{steps} plain P3M steps of the {n}-body adjoint workload ({el:.1f} s); "
                             f"the reference has no adjoint"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": (sum(f_ms) + sum(b_ms)) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "adjoint", "n_bodies": n, "rollout_steps": T,
                       "checkpoint_interval": ADJOINT_INTERVAL, "grid": "1024x512",
                       "boundary": "torus", "viewport_px": "2560x1440",
                       "step": "one forward rollout with checkpoints + its backward",
                       "l2": "flushed (256 MiB write) before every timed step",
                       "parallelism": "replicas" if args.gpus > 1 else "single"},
            "adjoint": {"plain_forward_ms": plain_ms, "checkpointed_forward_ms": f_avg,
                        "backward_ms": b_avg, "backward_over_plain_forward": b_avg / plain_ms,
                        "launch_velocity_px": list(ADJOINT_V0_PX), "target_px": list(ADJOINT_TARGET_PX),
                        "loss_px2": obj.loss, "grad_velocity_px": obj.grad_velocity_px.tolist(),
                        "fd_grad_velocity_px": fd.tolist(), "fd_h_px_per_s": ADJOINT_FD_H,
                        "fd_rel_err": fd_err, "fd_grad_other_h": fd_spread,
                        "fp64_reference": fp64},
            "roofline": None,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 32 * n,
                    "d2h_bytes_per_step": 32 * n, "steps": e2e_steps},
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    pipe.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=45)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default="lattice_scale",
                    choices=["plummer_walls", "uniform_torus", "lattice_scale", "lattice_scale_u32",
                             "batch", "adjoint"])
    ap.add_argument("--fp64-check", action="store_true",
                    help="adjoint workload: also run the FP64 reference adjoint on the host")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--bodies", type=int, default=None, help="override the workload's body count")
    ap.add_argument("--grid", default=None, help="override the workload's grid, WxH")
    ap.add_argument("--sims", type=int, default=None, help="batch: number of simulations")
    ap.add_argument("--batch-form", default="per_stage",
                    choices=["persistent", "per_stage", "per_simulation"],
                    help="batch --run-only: one persistent launch per step, one launch per "
                         "stage, or one step per simulation")
    ap.add_argument("--run-only", action="store_true",
                    help="run the initial pass and --steps steps untimed (a profiler's target)")
    ap.add_argument("--previews", type=int, default=0,
                    help="--run-only: then a fan of this many 1024-step aim previews")
    ap.add_argument("--no-plain", action="store_true",
                    help="lattice_scale: skip the 400k plummer_walls run beside it")
    ap.add_argument("--no-form-errors", action="store_true",
                    help="skip the force errors of the other deposit form and the oracle")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    ws, rank, local = dist_env()
    if args.run_only:
        run_only(args)
        return
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    if args.workload == "batch":
        run_batch(args, ws, rank, local)
        return
    if args.workload == "adjoint":
        run_adjoint(args, ws, rank, local)
        return
    run_b200(args, ws, rank, local)


if __name__ == "__main__":
    main()
