"""NUFFT throughput on B200: NU points/s of the 2D type-1 workload (1024^2 modes,
10^7 uniform points, eps 1e-5), one JSON line on rank 0.

A step is one type-1 execution on prepared points (sort done once by
set_points), the reference's execute_type1_gpu; `one_shot` adds the sort
(encode_type1_gpu). Inputs are resident in HBM; L2 is flushed with a 256 MiB
write between steps, outside the timed events. `e2e` runs the reference's C
interface with host buffers: pinned host -> device copies of points and
strengths, one-shot execution, device -> host copy of the modes, every step.

Every line reports its relative l2 error against FP64 direct sums over all
of its inputs, on >= 1,024 modes (type 1) or >= 10,000 points (type 2), or
every output where the workload is small, with `meets_eps` (rel-l2 <= eps)
and the reference's own test bound for that kind and dimension. The sums
come from the oracle's GPU checker (oracle/gpu_direct.py), which only
checks: nothing measured runs through it.

Secondary lines: the clustered variant of the headline workload; the small
2D configuration (64^2 modes, 10^5 points, eps 1e-6) with every output
checked and the CPU plan timed beside it; the batched sweep on one point set
(2D 512^2 modes, 2e6 points, B in {1, 16, 64, 256}, eps 1e-3 and 1e-6 on
CUDA cores and tensor cores; f64 and Df64 at eps 1e-9 and 1e-12); the 3D
radial configuration (256^3 modes, 49,999,872 points, eps 1e-5); 256 uneven
problems; 3D type-3 in f64; type-3 on small f32 grids.

`--impl reference` times the reference's CPU implementation of the path (its
CpuNufftPlan, restated under oracle/; the reference itself needs Rust and
wgpu, absent here) on the host cores, on all 10^7 points of the same plan:
its value is the execution on prepared points, the metric of the GPU arm's
value; the one-shot execution (with the sort) is reported beside it. With
torchrun, every rank runs the same workload on its own GPU (independent
replicas: weak scaling) and the slowest rank's time counts.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MODES = (1024, 1024)
POINTS = 10_000_000
EPS = 1e-5
SEED = 20240601
WORKLOAD = "2d_type1_modes1024x1024_M1e7_uniform_eps1e-5"
METRIC = "NU points/s (type-1 2D, 1024^2 modes, 1e7 uniform points, eps 1e-5, rel-l2 vs FP64 direct reported)"
UNIT = "points/s"
CHECK_MODES = 1024      # type-1 outputs checked against direct sums
CHECK_POINTS = 10_000   # type-2 outputs checked against direct sums
# The reference's relative-l2 test bounds (tests/gpu_nufft.rs:14-18,
# gpu_nufft_2d.rs:15-16, gpu_nufft_3d.rs:14-15, gpu_nufft_batch.rs:13-16,
# gpu_nufft_precision.rs:16-20, gpu_nufft_df64.rs:16-20, gpu_nufft_type3.rs:13-14).
REFERENCE_BOUND = {"1d": 4.0, "2d": 20.0, "3d": 32.0, "batch": 80.0, "f64": 20.0, "df64": 24.0, "type3": 100.0}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    for name in ("e2e", "cpu", "clustered", "small", "batched", "uneven", "radial", "f64", "type3", "peak"):
        p.add_argument(f"--no-{name}", action="store_true")
    return p.parse_args()


def make_inputs(rng_seed=SEED, count=POINTS):
    rng = np.random.default_rng(rng_seed)
    points = rng.uniform(-np.pi, np.pi, (count, 2)).astype(np.float32)
    strengths = (rng.standard_normal(count) + 1j * rng.standard_normal(count)).astype(np.complex64)
    return points, strengths


def cpu_nproc():
    threads = os.cpu_count() or 1
    try:
        threads = len(os.sched_getaffinity(0))
    except AttributeError:
        pass
    return threads


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_plan_timings(points, strengths, modes, eps, steps, warmup, kind=1):
    """Medians of the restated CPU plan over `steps` one-shot executions (after
    `warmup`): one-shot, point preparation, execution on prepared points; the
    same medians nufft_cpu_bench.rs:121-131 reports."""
    from oracle import native

    plan = native.CpuPlan(kind, modes, eps, precision="f32")
    threads = cpu_nproc()
    for _ in range(warmup):
        plan.execute(points, strengths, threads=threads)
    totals, stages = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        plan.execute(points, strengths, threads=threads, stage_seconds=stages)
        totals.append(time.perf_counter() - t0)
    return {"one_shot_s": statistics.median(totals), "prepare_s": statistics.median(s[0] for s in stages),
            "prepared_s": statistics.median(s[1] for s in stages), "threads": threads,
            "one_shot_total_s": sum(totals), "prepared_total_s": sum(s[1] for s in stages)}


def reference_arm(args):
    """The reference's CPU implementation (restated) on all points of the workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    points, strengths = make_inputs()
    t = cpu_plan_timings(points, strengths, MODES, EPS, args.steps, args.warmup)
    ms = 1e3 * t["prepared_total_s"] / args.steps
    value = POINTS / (ms / 1e3)
    sample = (f"all {POINTS:,} uniform points of the 1024^2-mode (2048^2 fine grid) eps 1e-5 plan per step; "
              f"value = execution on prepared points (median {1e3 * t['prepared_s']:.0f} ms), "
              f"one-shot with the sort {1e3 * t['one_shot_s']:.0f} ms; {t['threads']} threads of {cpu_model()}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded uniform)",
        "config": {"workload": WORKLOAD, "modes": list(MODES), "points": POINTS, "points_per_step": POINTS,
                   "eps": EPS},
        "one_shot": {"value": POINTS / t["one_shot_s"], "unit": UNIT, "ms_per_step": 1e3 * t["one_shot_s"]},
        "prepare_ms": 1e3 * t["prepare_s"],
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": t["threads"], "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().splitlines() if r.strip()]
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[5:9]) if "Active" in v
                          and "Not" not in v})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def max_over_ranks(values, device="cpu"):
    """The maximum of each value over all ranks (the slowest replica's time);
    the values themselves on a single process."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(values)
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def replica_throughput(world, units_per_replica, total_ms, steps):
    """Whole-job units/s of `world` independent replicas timed at the slowest one."""
    return world * units_per_replica / (total_ms / steps / 1e3)


class Runner:
    """Timing and accuracy helpers shared by every line."""

    def __init__(self, torch, w, args, world, rank, local):
        self.torch, self.w, self.args = torch, w, args
        self.world, self.rank, self.local = world, rank, local
        self.dev = f"cuda:{local}"
        self.flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=self.dev)
        self.stream = torch.cuda.current_stream()

    def barrier(self):
        import torch.distributed as dist

        if self.world > 1:
            dist.barrier()
        self.torch.cuda.synchronize()

    def timed(self, step_fn, steps, stream=None):
        """Total ms of `steps` calls, each bracketed by CUDA events on the
        launching stream after an L2 flush outside the events."""
        torch = self.torch
        stream = stream or self.stream
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for i in range(steps):
            with torch.cuda.stream(stream):
                self.flush.fill_(float(i))
            starts[i].record(stream)
            step_fn()
            ends[i].record(stream)
        torch.cuda.synchronize()
        return sum(s.elapsed_time(e) for s, e in zip(starts, ends))

    def measure(self, step_fn, units, steps, warmup):
        for _ in range(max(warmup, 1)):
            step_fn()
        self.barrier()
        total = self.timed(step_fn, steps)
        (total,) = max_over_ranks([total], self.dev)
        return {"value": replica_throughput(self.world, units, total, steps), "ms_per_step": total / steps}

    # Accuracy against FP64 direct sums (rank 0 only; None elsewhere).
    def check_type1(self, points, strengths, out, modes, eps, bound_key, vectors=4, count=CHECK_MODES, seed=1,
                    isign=1):
        if self.rank != 0:
            return None
        from oracle import gpu_direct

        n = int(np.prod(modes))
        select = np.sort(np.random.default_rng(seed).choice(n, min(count, n), replace=False))
        nb = min(vectors, strengths.shape[0] if strengths.dim() > 1 else 1)
        s = strengths.reshape(-1, points.shape[0])[:nb]
        ref = gpu_direct.direct_type1(points, s, modes, isign, select=select, device=self.dev)
        got = out.reshape(-1, n)[:nb][:, self.torch.as_tensor(select, device=self.dev)].cpu().numpy()
        return accuracy(got, ref, eps, bound_key, f"{len(select)} modes x {nb} vectors")

    def check_type2(self, points, coefficients, out, modes, eps, bound_key, vectors=4, count=CHECK_POINTS, seed=2,
                    isign=1):
        if self.rank != 0:
            return None
        from oracle import gpu_direct

        m = points.shape[0]
        n = int(np.prod(modes))
        pick = np.sort(np.random.default_rng(seed).choice(m, min(count, m), replace=False))
        nb = min(vectors, coefficients.reshape(-1, n).shape[0])
        ref = gpu_direct.direct_type2(points, coefficients.reshape(-1, n)[:nb], modes, isign, select=pick,
                                      device=self.dev)
        got = out.reshape(-1, m)[:nb][:, self.torch.as_tensor(pick, device=self.dev)].cpu().numpy()
        return accuracy(got, ref, eps, bound_key, f"{len(pick)} points x {nb} vectors")


def accuracy(got, ref, eps, bound_key, subset):
    rel = float(np.linalg.norm(got.astype(np.complex128) - ref) / np.linalg.norm(ref))
    bound = REFERENCE_BOUND[bound_key] * eps
    return {"rel_l2": rel, "eps": eps, "meets_eps": rel <= eps, "reference_bound": bound,
            "within_reference_bound": rel <= bound, "checked": subset}


def c_interface_e2e(r, points_h, strengths_h):
    """NU points/s of wgpu_nufftf_setpts + wgpu_nufftf_execute on pinned host arrays."""
    import ctypes

    from wgpunufft_b200 import _native

    torch = r.torch
    lib = _native.library()
    x = torch.from_numpy(np.ascontiguousarray(points_h[:, 0])).pin_memory()
    y = torch.from_numpy(np.ascontiguousarray(points_h[:, 1])).pin_memory()
    c = torch.from_numpy(strengths_h.view(np.float32)).pin_memory()
    f = torch.empty(MODES[0] * MODES[1] * 2, dtype=torch.float32).pin_memory()
    opts = _native.WgpuOpts()
    lib.wgpu_nufft_default_opts(ctypes.byref(opts))
    opts.adapter_index = torch.cuda.current_device() + 1
    plan = ctypes.c_void_p()
    modes = (ctypes.c_int64 * 2)(*MODES)
    code = lib.wgpu_nufftf_makeplan(1, 2, modes, 1, 1, EPS, ctypes.byref(plan), ctypes.byref(opts))
    if code != 0:
        return {"error": lib.wgpu_nufft_last_error().decode()}
    failures = []

    def step():
        rc = lib.wgpu_nufftf_setpts(plan, POINTS, x.data_ptr(), y.data_ptr(), None, 0, None, None, None)
        rc = rc or lib.wgpu_nufftf_execute(plan, c.data_ptr(), f.data_ptr())
        if rc:
            failures.append(lib.wgpu_nufft_last_error().decode())

    try:
        for _ in range(max(2, r.args.warmup)):
            step()
        r.barrier()
        e2e_ms = r.timed(step, r.args.steps)
    finally:
        lib.wgpu_nufftf_destroy(plan)
    if failures:
        return {"error": failures[0]}
    (e2e_ms,) = max_over_ranks([e2e_ms], r.dev)
    return {"value": replica_throughput(r.world, POINTS, e2e_ms, r.args.steps), "unit": UNIT,
            "ms_per_step": e2e_ms / r.args.steps,
            "h2d_bytes_per_step": POINTS * 4 * 2 + POINTS * 8, "d2h_bytes_per_step": MODES[0] * MODES[1] * 8,
            "path": "C interface wgpu_nufftf_setpts (per-axis f32, pinned host) + wgpu_nufftf_execute, "
                    "plan made once; host-to-device copies, stable bin sort, spread, FFT, deconvolution "
                    "and device-to-host copy inside every step"}


def stage_ms(stages, steps):
    return {k: round(v[0] / steps, 4) for k, v in stages.items()}


def clustered_line(r):
    """The clustered variant of the headline workload (8 centres, N(c, 0.01^2 I)
    wrapped), type 1 and type 2 on prepared points."""
    from wgpunufft_b200 import workloads

    torch, w = r.torch, r.w
    steps = max(1, min(r.args.steps, 5))
    pts = workloads.points("clustered", POINTS, 2, seed=SEED % 1000 + 21, device=r.dev)
    c = workloads.values(1, POINTS, seed=SEED % 1000 + 22, device=r.dev)
    n = MODES[0] * MODES[1]
    out = {"workload": "2d_modes1024x1024_M1e7_clustered_eps1e-5", "unit": UNIT}
    plan = w.NufftPlan.type1_gpu(w.NufftConfig(MODES, EPS))
    plan.set_points_gpu(pts)
    modes = torch.empty((1, n), dtype=torch.complex64, device=r.dev)
    out["type1"] = r.measure(lambda: plan.execute_gpu_batch(1, c, modes), POINTS, steps, r.args.warmup)
    out["type1"].update(r.check_type1(pts, c, modes, MODES, EPS, "2d") or {})
    del plan
    plan2 = w.NufftPlan.type2_gpu(w.NufftConfig(MODES, EPS))
    plan2.set_points_gpu(pts)
    f = workloads.values(1, n, seed=SEED % 1000 + 23, device=r.dev)
    vals = torch.empty((1, POINTS), dtype=torch.complex64, device=r.dev)
    out["type2"] = r.measure(lambda: plan2.execute_gpu_batch(1, f, vals), POINTS, steps, r.args.warmup)
    out["type2"].update(r.check_type2(pts, f, vals, MODES, EPS, "2d") or {})
    del plan2, pts, c, f, vals, modes
    torch.cuda.empty_cache()
    return out


def small_line(r):
    """The small 2D configuration: 64^2 modes, 10^5 uniform points, eps 1e-6,
    type 1 and type 2 with every output checked against FP64 direct sums over
    all points and modes, and the restated CPU plan timed on the same inputs."""
    torch, w = r.torch, r.w
    modes, count, eps = (64, 64), 100_000, 1e-6
    rng = np.random.default_rng(SEED + 11)
    pts_h = rng.uniform(-np.pi, np.pi, (count, 2)).astype(np.float32)
    c_h = (rng.standard_normal(count) + 1j * rng.standard_normal(count)).astype(np.complex64)
    f_h = (rng.standard_normal(64 * 64) + 1j * rng.standard_normal(64 * 64)).astype(np.complex64)
    pts = torch.from_numpy(pts_h).to(r.dev)
    c = torch.from_numpy(c_h).to(r.dev).reshape(1, -1)
    f = torch.from_numpy(f_h).to(r.dev).reshape(1, -1)
    steps = max(3, min(r.args.steps, 20))
    out = {"workload": "2d_modes64x64_M1e5_uniform_eps1e-6", "unit": UNIT}
    plan = w.NufftPlan.type1_gpu(w.NufftConfig(modes, eps))
    plan.set_points_gpu(pts)
    m1 = torch.empty((1, 4096), dtype=torch.complex64, device=r.dev)
    out["type1"] = r.measure(lambda: plan.execute_gpu_batch(1, c, m1), count, steps, r.args.warmup)
    out["type1"]["one_shot"] = r.measure(lambda: plan.encode_gpu_batch(1, pts, c, m1), count, steps, 1)["value"]
    out["type1"].update(r.check_type1(pts, c, m1, modes, eps, "2d", count=4096) or {})
    plan2 = w.NufftPlan.type2_gpu(w.NufftConfig(modes, eps))
    plan2.set_points_gpu(pts)
    v2 = torch.empty((1, count), dtype=torch.complex64, device=r.dev)
    out["type2"] = r.measure(lambda: plan2.execute_gpu_batch(1, f, v2), count, steps, r.args.warmup)
    out["type2"].update(r.check_type2(pts, f, v2, modes, eps, "2d", count=count) or {})
    if r.rank == 0 and not r.args.no_cpu:
        t1 = cpu_plan_timings(pts_h, c_h, modes, eps, 5, 1, kind=1)
        t2 = cpu_plan_timings(pts_h, f_h, modes, eps, 5, 1, kind=2)
        out["cpu_plan"] = {"type1_prepared": count / t1["prepared_s"], "type1_one_shot": count / t1["one_shot_s"],
                           "type2_prepared": count / t2["prepared_s"], "type2_one_shot": count / t2["one_shot_s"],
                           "threads": t1["threads"], "unit": UNIT}
    del plan, plan2
    return out


BATCH_MODES = (512, 512)
BATCH_POINTS = 2_000_000


def batched_sweep(r):
    """One point set (2D 512^2 modes, 2e6 uniform points), B vectors: f32 type 1
    and type 2 on CUDA cores and on tensor cores (3xTF32), eps 1e-3 and 1e-6,
    B in {1, 16, 64, 256}; f64 and Df64 at eps 1e-9 and 1e-12 for B in {1, 16}.
    NU points/s counts points x vectors."""
    from wgpunufft_b200 import workloads

    torch, w = r.torch, r.w
    steps = max(1, min(r.args.steps, 5))
    pts = workloads.points("uniform", BATCH_POINTS, 2, seed=SEED % 1000 + 4, device=r.dev)
    n = BATCH_MODES[0] * BATCH_MODES[1]
    result = {"workload": "2d_modes512x512_M2e6_uniform", "unit": "NU points/s (points x vectors)"}
    for eps in (1e-3, 1e-6):
        for batch in (1, 16, 64, 256):
            c = workloads.values(batch, BATCH_POINTS, seed=batch, device=r.dev)
            modes = torch.empty((batch, n), dtype=torch.complex64, device=r.dev)
            entry = {}
            for name, method in (("tensor_cores", w.SpreadMethod.TENSOR_CORES),
                                 ("cuda_cores", w.SpreadMethod.CUDA_CORES)):
                plan = w.NufftPlan.type1_gpu(w.NufftConfig(BATCH_MODES, eps, batch=batch, spread_method=method))
                plan.set_points_gpu(pts)
                plan.stage_timing(True)
                item = r.measure(lambda: plan.execute_gpu_batch(batch, c, modes), BATCH_POINTS * batch, steps,
                                 r.args.warmup)
                stages = plan.stage_report()
                plan.stage_timing(False)
                item["spread_ms"] = round(stages.get("spread", (0.0, 1))[0] / (steps + max(r.args.warmup, 1)), 4)
                item.update(r.check_type1(pts, c, modes, BATCH_MODES, eps, "batch", seed=batch) or {})
                entry[f"type1_{name}"] = item
                del plan
            entry["tensor_over_cuda_cores"] = entry["type1_tensor_cores"]["value"] / entry["type1_cuda_cores"]["value"]
            del c, modes
            f = workloads.values(batch, n, seed=1000 + batch, device=r.dev)
            vals = torch.empty((batch, BATCH_POINTS), dtype=torch.complex64, device=r.dev)
            for name, method in (("tensor_cores", w.SpreadMethod.TENSOR_CORES),
                                 ("cuda_cores", w.SpreadMethod.CUDA_CORES)):
                plan2 = w.NufftPlan.type2_gpu(w.NufftConfig(BATCH_MODES, eps, batch=batch, spread_method=method))
                plan2.set_points_gpu(pts)
                plan2.stage_timing(True)
                item2 = r.measure(lambda: plan2.execute_gpu_batch(batch, f, vals), BATCH_POINTS * batch, steps,
                                  r.args.warmup)
                stages = plan2.stage_report()
                plan2.stage_timing(False)
                item2["interpolation_ms"] = round(
                    stages.get("interpolation", (0.0, 1))[0] / (steps + max(r.args.warmup, 1)), 4)
                item2.update(r.check_type2(pts, f, vals, BATCH_MODES, eps, "batch", seed=batch) or {})
                entry[f"type2_{name}"] = item2
                del plan2
            entry["type2_tensor_over_cuda_cores"] = (entry["type2_tensor_cores"]["value"] /
                                                     entry["type2_cuda_cores"]["value"])
            del f, vals
            torch.cuda.empty_cache()
            result[f"eps{eps:g}_B{batch}"] = entry
    pts64 = pts.double()
    for precision, tag in ((w.Precision.F64, "f64"), (w.Precision.DF64, "df64")):
        for eps in (1e-9, 1e-12):
            for batch in (1, 16):
                c = workloads.values(batch, BATCH_POINTS, seed=batch + 7, device=r.dev).to(torch.complex128)
                f = workloads.values(batch, n, seed=batch + 8, device=r.dev).to(torch.complex128)
                entry = {}
                if precision == w.Precision.DF64:
                    p_in, c_in, f_in = to_df64(torch, pts64), to_df64(torch, c), to_df64(torch, f)
                else:
                    p_in, c_in, f_in = pts64, c, f
                for kind in (1, 2):
                    config = w.NufftConfig(BATCH_MODES, eps, batch=batch, precision=precision)
                    plan = (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(config)
                    outputs = n if kind == 1 else BATCH_POINTS
                    if precision == w.Precision.DF64:
                        # (hi, lo) float pairs of the real and imaginary parts.
                        out = torch.empty((batch, 4 * outputs), dtype=torch.float32, device=r.dev)
                    else:
                        out = torch.empty((batch, outputs), dtype=torch.complex128, device=r.dev)
                    plan.set_points_gpu(p_in)
                    inputs = c_in if kind == 1 else f_in
                    item = r.measure(lambda: plan.execute_gpu_batch(batch, inputs, out), BATCH_POINTS * batch,
                                     steps, r.args.warmup)
                    item["kernel_width"] = plan.kernel_width()
                    got = from_df64(torch, out) if precision == w.Precision.DF64 else out
                    if kind == 1:
                        item.update(r.check_type1(pts64, c, got, BATCH_MODES, eps, tag, seed=batch) or {})
                    else:
                        item.update(r.check_type2(pts64, f, got, BATCH_MODES, eps, tag, seed=batch) or {})
                    entry[f"type{kind}"] = item
                    del plan, out
                result[f"{tag}_eps{eps:g}_B{batch}"] = entry
                del c, f, p_in, c_in, f_in
                torch.cuda.empty_cache()
    del pts, pts64
    torch.cuda.empty_cache()
    return result


def tensor_peak_line(r):
    """tcgen05.mma throughput on this GPU (b200nufft_tf32_peak: every SM
    issuing back-to-back M=128 MMAs from one elected lane, 16 straight-line
    MMAs per block): kind::tf32 (K=8) at N=256 is the dense tf32 peak, N=16
    and 32 the narrow MMAs of the tensor-core interpolation; kind::f16 (K=16)
    beside it. Cycles per MMA come from the SM clock counter of CTA 0 (issue
    plus drain), independent of the clock frequency."""
    import ctypes

    from wgpunufft_b200 import _native

    lib = _native.library()
    sms = r.torch.cuda.get_device_properties(r.local).multi_processor_count
    out = {"unit": "TFLOP/s", "sms": sms}
    for kind, f16, k in (("tf32", 0, 8), ("f16", 1, 16)):
        for n in (256, 32, 16):
            for where, a_tmem in (("a_smem", 0), ("a_tmem", 1)):
                iters = 40000
                ms = ctypes.c_float(0.0)
                cycles = (ctypes.c_uint64 * 2)()
                status = lib.b200nufft_tf32_peak(n, a_tmem, iters, 1, f16, 16, 0, ctypes.byref(ms), cycles)
                key = f"{kind}_n{n}_{where}"
                if status != 0 or ms.value <= 0:
                    out[key] = {"status": status}
                    continue
                flops = 2.0 * 128 * n * k * iters * sms
                out[key] = {"tflops": flops / (ms.value / 1e3) / 1e12, "ms": ms.value,
                            "cycles_per_mma": cycles[1] / iters}
    return out


def to_df64(torch, x):
    """Double-float storage of an f64 (or c128) tensor: (hi, lo) f32 pairs per scalar."""
    real = torch.view_as_real(x) if x.is_complex() else x
    hi = real.to(torch.float32)
    lo = (real - hi.to(torch.float64)).to(torch.float32)
    return torch.stack([hi, lo], dim=-1).contiguous()


def from_df64(torch, pairs):
    """The complex128 values of Df64 output storage (hi, lo pairs of re and im)."""
    p = torch.view_as_real(pairs) if pairs.is_complex() else pairs
    p = p.reshape(p.shape[0], -1, 2, 2).to(torch.float64)
    v = p[..., 0] + p[..., 1]
    return torch.complex(v[..., 0], v[..., 1])


def radial_3d_line(r):
    """The 3D configuration: 256^3 modes, 4096 radial spokes x 12207 samples
    (49,999,872 points), eps 1e-5; type 1 and type 2 on prepared points."""
    from wgpunufft_b200 import workloads

    torch, w = r.torch, r.w
    modes, count, eps, dist = workloads.CASES["radial"]
    pts = workloads.points(dist, count, 3, seed=SEED % 1000 + 31, device=r.dev)
    c = workloads.values(1, count, seed=SEED % 1000 + 32, device=r.dev)
    n = modes[0] * modes[1] * modes[2]
    result = {"workload": "3d_modes256^3_M49999872_radial_eps1e-5", "unit": UNIT}
    steps = max(1, min(r.args.steps, 5))
    plan = w.NufftPlan.type1_gpu(w.NufftConfig(modes, eps))
    plan.set_points_gpu(pts)
    out = torch.empty((1, n), dtype=torch.complex64, device=r.dev)
    plan.stage_timing(True)
    item = r.measure(lambda: plan.execute_gpu_batch(1, c, out), count, steps, r.args.warmup)
    item["stages_ms_per_step"] = stage_ms(plan.stage_report(), steps + max(r.args.warmup, 1))
    plan.stage_timing(False)
    item.update(r.check_type1(pts, c, out, modes, eps, "3d") or {})
    result["type1"] = item
    del plan, out
    torch.cuda.empty_cache()
    plan2 = w.NufftPlan.type2_gpu(w.NufftConfig(modes, eps))
    plan2.set_points_gpu(pts)
    f = workloads.values(1, n, seed=SEED % 1000 + 33, device=r.dev)
    vals = torch.empty((1, count), dtype=torch.complex64, device=r.dev)
    item2 = r.measure(lambda: plan2.execute_gpu_batch(1, f, vals), count, steps, r.args.warmup)
    item2.update(r.check_type2(pts, f, vals, modes, eps, "3d") or {})
    result["type2"] = item2
    del plan2, f, vals, pts, c
    torch.cuda.empty_cache()
    return result


def type3_line(r):
    """3D type 3 in f64: 10^6 sources uniform in [-1, 1]^3 to 10^6 targets
    uniform in [-200, 200]^3, eps 1e-9, checked on 1,000 targets; and f32 type
    3 on small outer grids (10^6 sources in [-1, 1]^d to 10^6 targets in
    [-30, 30]^d, eps 1e-6, d = 1 and 2), the regime of the reference's dense
    small-grid spreader (src/gpu_dense_spread.rs:68-78)."""
    torch, w = r.torch, r.w
    count = 1_000_000
    g = torch.Generator(device=r.dev)
    g.manual_seed(SEED + 51)
    src = (torch.rand((count, 3), generator=g, device=r.dev, dtype=torch.float64) * 2 - 1).contiguous()
    tgt = (torch.rand((count, 3), generator=g, device=r.dev, dtype=torch.float64) * 400 - 200).contiguous()
    c = torch.complex(torch.randn((1, count), generator=g, device=r.dev, dtype=torch.float64),
                      torch.randn((1, count), generator=g, device=r.dev, dtype=torch.float64))
    plan = w.NufftType3Plan(w.NufftType3Config(((-1.0, 1.0),) * 3, ((-200.0, 200.0),) * 3, eps=1e-9))
    out = torch.empty((1, count), dtype=torch.complex128, device=r.dev)
    steps = max(1, min(r.args.steps, 3))
    plan.set_points_gpu(src, tgt)
    result = {"workload": "3d_type3_f64_src1e6_in[-1,1]^3_tgt1e6_in[-200,200]^3_eps1e-9", "unit": UNIT,
              "note": "points/s counts sources (= targets)"}
    result.update(r.measure(lambda: plan.execute_gpu_batch(1, c, out), count, steps, r.args.warmup))
    result["with_set_points"] = r.measure(lambda: plan.encode_gpu_batch(1, src, c, tgt, out), count, steps, 1)
    if r.rank == 0:
        from oracle import gpu_direct

        pick = np.sort(np.random.default_rng(14).choice(count, 1000, replace=False))
        ref = gpu_direct.direct_type3(src, c, tgt, 1, select=pick, device=r.dev)
        got = out[:, torch.as_tensor(pick, device=r.dev)].cpu().numpy()
        result.update(accuracy(got, ref, 1e-9, "type3", "1000 targets"))
    del plan, out, src, tgt, c
    torch.cuda.empty_cache()
    lines = {}
    for d in (1, 2):
        g = torch.Generator(device=r.dev)
        g.manual_seed(SEED + 60 + d)
        src = (torch.rand((count, d), generator=g, device=r.dev) * 2 - 1).contiguous()
        tgt = (torch.rand((count, d), generator=g, device=r.dev) * 60 - 30).contiguous()
        c = torch.complex(torch.randn((1, count), generator=g, device=r.dev),
                          torch.randn((1, count), generator=g, device=r.dev))
        config = w.NufftType3Config(((-1.0, 1.0),) * d, ((-30.0, 30.0),) * d, eps=1e-6, precision=w.Precision.F32)
        plan = w.NufftType3Plan(config)
        out = torch.empty((1, count), dtype=torch.complex64, device=r.dev)
        plan.set_points_gpu(src, tgt)
        line = {"workload": f"{d}d_type3_f32_src1e6_in[-1,1]^{d}_tgt1e6_in[-30,30]^{d}_eps1e-6", "unit": UNIT,
                "outer_grid": list(plan.info().outer_shape[:d])}
        line.update(r.measure(lambda: plan.execute_gpu_batch(1, c, out), count, steps, r.args.warmup))
        if r.rank == 0:
            from oracle import gpu_direct

            pick = np.sort(np.random.default_rng(15 + d).choice(count, 1000, replace=False))
            ref = gpu_direct.direct_type3(src, c, tgt, 1, select=pick, device=r.dev)
            got = out[:, torch.as_tensor(pick, device=r.dev)].cpu().numpy()
            line.update(accuracy(got, ref, 1e-6, "type3", "1000 targets"))
        lines[f"{d}d"] = line
        del plan, out, src, tgt, c
    result["small_outer_grids_f32"] = lines
    torch.cuda.empty_cache()
    return result


def uneven_problems_line(r):
    """256 independent type-1 problems of uneven sizes (2D/3D, 64^2..256^2 and
    32^3..64^3 modes, 1e3..1e6 points, uniform or clustered, eps 1e-6), one
    plan each with its points set: all executions issued one after another
    (eager) and replayed from one captured CUDA graph."""
    from wgpunufft_b200 import workloads

    torch, w = r.torch, r.w
    problems = workloads.uneven_problems(256, seed=SEED % 1000)
    stream = torch.cuda.Stream()
    plans, outs = [], []
    with torch.cuda.stream(stream):
        for modes, p, c in problems:
            plan = w.NufftPlan.type1_gpu(w.NufftConfig(modes, 1e-6))
            plan.set_points_gpu(p, stream=stream)
            out = torch.empty((1, int(np.prod(modes))), dtype=torch.complex64, device=r.dev)
            plan.execute_gpu_batch(1, c, out, stream=stream)
            plans.append(plan)
            outs.append(out)
        stream.synchronize()

        def run_all():
            for plan, (modes, p, c), out in zip(plans, problems, outs):
                plan.execute_gpu_batch(1, c, out, stream=stream)

        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            run_all()
        stream.synchronize()
        steps = max(1, min(r.args.steps, 5))
        for _ in range(max(2, r.args.warmup)):
            run_all()
            graph.replay()
        r.barrier()
        eager_ms = r.timed(run_all, steps, stream)
        graph_ms = r.timed(graph.replay, steps, stream)
        # The same problems as one batch: one persistent spreading launch over
        # every problem's tile parts, then per-problem folds, FFTs and
        # deconvolutions on forked streams.
        batch = w.NufftBatch(plans)
        strengths = [c for _, _, c in problems]
        batch_outs = [torch.empty_like(o) for o in outs]

        def run_batch():
            batch.execute(strengths, batch_outs, stream=stream)

        run_batch()
        stream.synchronize()
        identical = all(torch.equal(a.view(torch.int32), b.view(torch.int32)) for a, b in zip(batch_outs, outs))
        batch_graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(batch_graph, stream=stream):
            run_batch()
        for _ in range(max(2, r.args.warmup)):
            run_batch()
            batch_graph.replay()
        r.barrier()
        batch_ms = r.timed(run_batch, steps, stream)
        batch_graph_ms = r.timed(batch_graph.replay, steps, stream)
    del graph, batch_graph, batch
    eager_ms, graph_ms, batch_ms, batch_graph_ms = max_over_ranks([eager_ms, graph_ms, batch_ms, batch_graph_ms],
                                                                  r.dev)
    total_points = sum(int(p.shape[0]) for _, p, _ in problems)
    return {"problems": len(problems), "points": total_points, "eps": 1e-6, "unit": UNIT,
            "graph": {"value": replica_throughput(r.world, total_points, graph_ms, steps),
                      "ms_per_step": graph_ms / steps},
            "eager": {"value": replica_throughput(r.world, total_points, eager_ms, steps),
                      "ms_per_step": eager_ms / steps},
            "persistent_batch": {"value": replica_throughput(r.world, total_points, batch_ms, steps),
                                 "ms_per_step": batch_ms / steps, "same_bits_as_plans": identical},
            "persistent_batch_graph": {"value": replica_throughput(r.world, total_points, batch_graph_ms, steps),
                                       "ms_per_step": batch_graph_ms / steps},
            "note": "one plan per problem (prepared points); a step executes all 256"}


def profile_traffic():
    """DRAM bytes per spread launch from the committed ncu capture of the same
    launch (profiles/spread_tiles_2d_1024_M1e7.md), if present."""
    path = ROOT / "profiles" / "spread_tiles_2d_1024_M1e7.md"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def compact(value, digits=4):
    if isinstance(value, float):
        return float(f"{value:.{digits}g}")
    if isinstance(value, dict):
        return {k: compact(v, digits) for k, v in value.items()}
    if isinstance(value, list):
        return [compact(v, digits) for v in value]
    return value


def summary_of(line):
    """The figures a reader needs first, kept short (the end of the line)."""
    s = {}
    if line.get("type2"):
        s["type2"] = {k: line["type2"].get(k) for k in ("value", "rel_l2", "meets_eps")}
    if line.get("one_shot"):
        s["one_shot"] = line["one_shot"].get("value")
    c = line.get("clustered")
    if c:
        s["clustered"] = {k: {q: c[k].get(q) for q in ("value", "rel_l2", "meets_eps")} for k in ("type1", "type2")}
    sm = line.get("small_2d")
    if sm:
        s["small_2d"] = {k: {q: sm[k].get(q) for q in ("value", "rel_l2", "meets_eps")} for k in ("type1", "type2")}
    b = line.get("batched")
    if b:
        s["batched"] = {}
        for key, entry in b.items():
            if not isinstance(entry, dict):
                continue
            s["batched"][key] = {k: [entry[k].get("value"), entry[k].get("rel_l2")] for k in entry
                                 if isinstance(entry[k], dict)}
    rad = line.get("radial_3d")
    if rad:
        s["radial_3d"] = {k: {q: rad[k].get(q) for q in ("value", "rel_l2", "meets_eps")} for k in ("type1", "type2")}
    u = line.get("uneven_problems")
    if u:
        s["uneven_ms"] = {k: u[k]["ms_per_step"] for k in ("graph", "persistent_batch", "persistent_batch_graph")
                          if k in u}
    t3 = line.get("type3")
    if t3:
        s["type3_f64"] = {q: t3.get(q) for q in ("value", "rel_l2")}
    return compact(s, 3)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    import wgpunufft_b200 as w

    r = Runner(torch, w, args, world, rank, local)
    dev = r.dev
    points_h, strengths_h = make_inputs()
    points = torch.from_numpy(points_h).to(dev)
    strengths = torch.from_numpy(strengths_h.view(np.float32)).to(dev).view(torch.complex64)
    config = w.NufftConfig(MODES, EPS)
    plan = w.NufftPlan.type1_gpu(config, device=local)
    out = torch.empty(config.mode_count(), dtype=torch.complex64, device=dev)

    # Warm-up: plan scratch, cuFFT plan, the sort.
    plan.set_points_gpu(points)
    for _ in range(args.warmup):
        plan.execute_type1_gpu(strengths, out)
        plan.encode_type1_gpu(points, strengths, out)
    plan.synchronize()

    # Prepared executions (the headline value), with stage events.
    plan.set_points_gpu(points)
    plan.synchronize()
    plan.stage_timing(True)
    plan.stage_report()
    launches0 = w.launch_count()
    r.barrier()
    with ClockSampler(local) as clocks:
        total_ms = r.timed(lambda: plan.execute_type1_gpu(strengths, out), args.steps)
        launches = w.launch_count() - launches0
        stages = plan.stage_report()
        plan.stage_timing(False)
        one_shot_ms = r.timed(lambda: plan.encode_type1_gpu(points, strengths, out), args.steps)
    r.barrier()
    clock_summary = clocks.summary()
    total_ms, one_shot_ms = max_over_ranks([total_ms, one_shot_ms], dev)
    ms = total_ms / args.steps
    value = replica_throughput(world, POINTS, total_ms, args.steps)
    one_shot = replica_throughput(world, POINTS, one_shot_ms, args.steps)
    plan.set_points_gpu(points)
    plan.execute_type1_gpu(strengths, out)
    plan.synchronize()
    headline_accuracy = r.check_type1(points, strengths, out, MODES, EPS, "2d")

    # Type 2 on the same points (reported beside the headline, same timing rules).
    plan2 = w.NufftPlan.type2_gpu(config, device=local)
    coefficients = torch.complex(torch.randn(config.mode_count(), device=dev),
                                 torch.randn(config.mode_count(), device=dev))
    values = torch.empty(POINTS, dtype=torch.complex64, device=dev)
    plan2.set_points_gpu(points)
    for _ in range(args.warmup):
        plan2.execute_type2_gpu(coefficients, values)
    plan2.synchronize()
    plan2.stage_timing(True)
    plan2.stage_report()
    type2_ms = r.timed(lambda: plan2.execute_type2_gpu(coefficients, values), args.steps)
    stages2 = plan2.stage_report()
    plan2.stage_timing(False)
    type2_one_shot_ms = r.timed(lambda: plan2.encode_type2_gpu(points, coefficients, values), args.steps)
    type2_ms, type2_one_shot_ms = max_over_ranks([type2_ms, type2_one_shot_ms], dev)
    plan2.set_points_gpu(points)
    plan2.execute_type2_gpu(coefficients, values)
    plan2.synchronize()
    type2 = {"value": replica_throughput(world, POINTS, type2_ms, args.steps), "unit": UNIT,
             "ms_per_step": type2_ms / args.steps,
             "one_shot_value": replica_throughput(world, POINTS, type2_one_shot_ms, args.steps),
             "stages_ms_per_step": stage_ms(stages2, args.steps)}
    type2.update(r.check_type2(points, coefficients, values, MODES, EPS, "2d") or {})
    del plan2, coefficients, values

    e2e = None if args.no_e2e else c_interface_e2e(r, points_h, strengths_h)
    clustered = None if args.no_clustered else clustered_line(r)
    small = None if args.no_small else small_line(r)
    batched = None if args.no_batched else batched_sweep(r)
    uneven = None if args.no_uneven else uneven_problems_line(r)
    radial = None if args.no_radial else radial_3d_line(r)
    type3 = None if args.no_type3 else type3_line(r)
    tensor_peak = None if args.no_peak else tensor_peak_line(r)

    if rank == 0:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
        hbm = peaks.get("hbm_gbs", 6650.0)
        spread_ms, spread_launches = stages.get("spread", (0.0, 0))
        per_launch_ms = spread_ms / max(spread_launches, 1)
        fine = plan.fine_grid_shape()
        # Type-1 spread bytes (coordinates as the 16-byte prepared windows, the
        # permutation word, the strength, and the padded tiles written).
        algorithmic = POINTS * (4 * 2 + 8 + 4) + fine[0] * fine[1] * 8
        achieved = algorithmic / (per_launch_ms / 1e3) / 1e9 if per_launch_ms > 0 else None
        roofline = {"bound": "hbm", "kernel": "spread_tiles_kernel<2,6>", "achieved": achieved, "peak": hbm,
                    "unit": "GB/s", "frac": achieved / hbm if achieved else None,
                    "traffic": profile_traffic(),
                    "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of this "
                                      "launch at this workload (profiles/spread_tiles_2d_1024_M1e7.md), not this run",
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650 GB/s",
                    "algorithmic_bytes_per_launch": algorithmic, "launch_ms": per_launch_ms}
        cpu = None
        if not args.no_cpu:
            t = cpu_plan_timings(points_h, strengths_h, MODES, EPS, 3, 1)
            cpu = {"value": POINTS / t["prepared_s"], "unit": UNIT, "cores": t["threads"], "kind": "port",
                   "sample": f"all {POINTS:,} points, same plan; restated CpuNufftPlan, execution on prepared "
                             f"points (median of 3: {1e3 * t['prepared_s']:.0f} ms; one-shot with the sort "
                             f"{1e3 * t['one_shot_s']:.0f} ms) on {t['threads']} threads of {cpu_model()}",
                   "one_shot_value": POINTS / t["one_shot_s"]}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded uniform points, N(0,1) strengths)",
            "config": {"workload": WORKLOAD, "modes": list(MODES), "points": POINTS, "eps": EPS, "batch": 1,
                       "fine_grid": list(fine), "kernel_width": plan.kernel_width(),
                       "l2": "flushed between steps by a 256 MiB write outside the timed events",
                       "parallelism": f"replicas x{world}"},
            "batched": compact(batched) if batched else None,
            "clustered": compact(clustered) if clustered else None,
            "small_2d": compact(small) if small else None,
            "radial_3d": compact(radial) if radial else None,
            "uneven_problems": compact(uneven) if uneven else None,
            "type3": compact(type3) if type3 else None,
            "tf32_tensor_peak": compact(tensor_peak) if tensor_peak else None,
            "stages_ms_per_step": stage_ms(stages, args.steps),
            "type2": compact(type2),
            "one_shot": {"value": one_shot, "unit": UNIT, "ms_per_step": one_shot_ms / args.steps,
                         "note": "set_points (stable bin sort) + execute per step"},
            "accuracy": headline_accuracy,
            "rel_l2": headline_accuracy["rel_l2"] if headline_accuracy else None,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clock_summary,
        }
        line["summary"] = summary_of(line)
        print(json.dumps(line, separators=(",", ":")), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
