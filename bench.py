"""NUFFT throughput on B200: NU points/s of the 2D type-1 workload (1024^2 modes,
10^7 uniform points, eps 1e-5), one JSON line on rank 0.

A step is one type-1 execution on prepared points (sort done once by
set_points), the reference's execute_type1_gpu; `one_shot` adds the sort
(encode_type1_gpu). Inputs are resident in HBM; L2 is flushed with a 256 MiB
write between steps, outside the timed events. `e2e` runs the public API with
host buffers: pinned host -> device copies of points and strengths, one-shot
execution, device -> host copy of the modes, every step. `--impl reference`
times the reference's CPU plan (its restatement under oracle/; the reference
itself needs Rust and wgpu, absent here) on the host cores. With torchrun,
every rank runs the same workload on its own GPU (independent replicas: weak
scaling) and the slowest rank's time counts.
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
CPU_SAMPLE = 1_000_000


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-uneven", action="store_true")
    p.add_argument("--no-radial", action="store_true")
    p.add_argument("--no-f64", action="store_true")
    p.add_argument("--no-type3", action="store_true")
    return p.parse_args()


def make_inputs(rng_seed=SEED, count=POINTS):
    rng = np.random.default_rng(rng_seed)
    points = rng.uniform(-np.pi, np.pi, (count, 2)).astype(np.float32)
    strengths = (rng.standard_normal(count) + 1j * rng.standard_normal(count)).astype(np.complex64)
    return points, strengths


def cpu_plan_throughput(points, strengths, repeats=3):
    """Median NU points/s of the restated CPU plan (one-shot execution) over `repeats` runs."""
    from oracle import native

    plan = native.CpuPlan(1, MODES, EPS, precision="f32")
    threads = os.cpu_count() or 1
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        plan.execute(points, strengths, threads=threads)
        times.append(time.perf_counter() - t0)
    return len(points) / statistics.median(times), threads, statistics.median(times)


def reference_arm(args):
    """The reference's CPU implementation (restated) on a bounded sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import native

    points, strengths = make_inputs(count=CPU_SAMPLE)
    plan = native.CpuPlan(1, MODES, EPS, precision="f32")
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        plan.execute(points, strengths, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        plan.execute(points, strengths, threads=threads)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    value = CPU_SAMPLE / (ms / 1e3)
    sample = (f"{CPU_SAMPLE:,} of the {POINTS:,} uniform points per step on the same 1024^2-mode "
              f"(2048^2 fine grid) eps 1e-5 plan; one-shot execution incl. sort")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded uniform)",
        "config": {"workload": WORKLOAD, "modes": list(MODES), "points_per_step": CPU_SAMPLE, "eps": EPS},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
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


def c_interface_e2e(w, torch, points_h, strengths_h, timed, barrier, world, dev, args):
    """NU points/s of wgpu_nufftf_setpts + wgpu_nufftf_execute on pinned host arrays."""
    import ctypes

    from wgpunufft_b200 import _native

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
        for _ in range(2):
            step()
        barrier()
        e2e_ms = timed(step, args.steps)
    finally:
        lib.wgpu_nufftf_destroy(plan)
    if failures:
        return {"error": failures[0]}
    (e2e_ms,) = max_over_ranks([e2e_ms], dev)
    return {"value": replica_throughput(world, POINTS, e2e_ms, args.steps), "unit": UNIT,
            "ms_per_step": e2e_ms / args.steps,
            "h2d_bytes_per_step": POINTS * 4 * 2 + POINTS * 8, "d2h_bytes_per_step": MODES[0] * MODES[1] * 8,
            "path": "C interface wgpu_nufftf_setpts (per-axis f32, pinned host) + wgpu_nufftf_execute, "
                    "plan made once; host-to-device copies, stable bin sort, spread, FFT, deconvolution "
                    "and device-to-host copy inside every step"}


BATCH_MODES = (512, 512)
BATCH_POINTS = 2_000_000
BATCH_EPS = 1e-6


def batched_comparison(w, torch, timed, barrier, world, dev, args, rank):
    """Type-1 NU points/s (points x vectors) of 64 and 256 vectors sharing one
    point set, tensor cores (3xTF32) against CUDA cores, plus rel-l2 against
    FP64 direct sums on 8 modes x 4 vectors."""
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 4)
    pts = (torch.rand((BATCH_POINTS, 2), generator=g, device=dev) * (2 * np.pi) - np.pi).float().contiguous()
    result = {"workload": "2d_type1_modes512x512_M2e6_uniform_eps1e-6", "modes": list(BATCH_MODES),
              "points": BATCH_POINTS, "eps": BATCH_EPS, "unit": "NU points/s (points x vectors)"}
    steps = max(1, min(args.steps, 5))
    select = np.random.default_rng(3).choice(BATCH_MODES[0] * BATCH_MODES[1], 8, replace=False)
    pts_h = pts.cpu().numpy().astype(np.float64) if rank == 0 else None
    for batch in (64, 256):
        c = torch.complex(torch.randn((batch, BATCH_POINTS), generator=g, device=dev),
                          torch.randn((batch, BATCH_POINTS), generator=g, device=dev))
        out = torch.empty((batch, BATCH_MODES[0] * BATCH_MODES[1]), dtype=torch.complex64, device=dev)
        entry = {}
        for name, method in (("tensor_cores", w.SpreadMethod.TENSOR_CORES), ("cuda_cores", w.SpreadMethod.CUDA_CORES)):
            plan = w.NufftPlan.type1_gpu(w.NufftConfig(BATCH_MODES, BATCH_EPS, batch=batch, spread_method=method))
            plan.set_points_gpu(pts)
            for _ in range(max(1, args.warmup)):
                plan.execute_gpu_batch(batch, c, out)
            barrier()
            plan.stage_timing(True)
            plan.stage_report()
            total = timed(lambda: plan.execute_gpu_batch(batch, c, out), steps)
            stages = plan.stage_report()
            plan.stage_timing(False)
            (total,) = max_over_ranks([total], dev)
            ms = total / steps
            item = {"value": replica_throughput(world, BATCH_POINTS * batch, total, steps), "ms_per_step": ms,
                    "stages_ms_per_step": {k: v[0] / steps for k, v in stages.items()}}
            if rank == 0:
                from oracle import native

                got = out[:4].cpu().numpy()[:, select]
                ref = native.direct_type1(pts_h, c[:4].cpu().numpy().astype(np.complex128), BATCH_MODES,
                                          select=select)
                item["rel_l2"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
            entry[name] = item
            del plan
        # Type 2 on the same points: modes of every vector to the points.
        plan2 = w.NufftPlan.type2_gpu(w.NufftConfig(BATCH_MODES, BATCH_EPS, batch=batch))
        plan2.set_points_gpu(pts)
        f = torch.complex(torch.randn((batch, BATCH_MODES[0] * BATCH_MODES[1]), generator=g, device=dev),
                          torch.randn((batch, BATCH_MODES[0] * BATCH_MODES[1]), generator=g, device=dev))
        vals = torch.empty((batch, BATCH_POINTS), dtype=torch.complex64, device=dev)
        for _ in range(max(1, args.warmup)):
            plan2.execute_gpu_batch(batch, f, vals)
        barrier()
        total2 = timed(lambda: plan2.execute_gpu_batch(batch, f, vals), steps)
        (total2,) = max_over_ranks([total2], dev)
        item2 = {"value": replica_throughput(world, BATCH_POINTS * batch, total2, steps), "ms_per_step": total2 / steps,
                 "engine": "CUDA cores, bin regions staged in shared memory"}
        if rank == 0:
            from oracle import native

            pick = np.random.default_rng(4).choice(BATCH_POINTS, 64, replace=False)
            ref2 = native.direct_type2(pts_h[pick], f[:4].cpu().numpy().astype(np.complex128), BATCH_MODES)
            got2 = vals[:4].cpu().numpy()[:, pick]
            item2["rel_l2"] = float(np.linalg.norm(got2 - ref2) / np.linalg.norm(ref2))
        entry["type2"] = item2
        del plan2, f, vals
        entry["speedup_tensor_over_cuda_cores"] = entry["tensor_cores"]["value"] / entry["cuda_cores"]["value"]
        spread_ms = entry["tensor_cores"]["stages_ms_per_step"].get("spread", 0.0)
        useful = 4.0 * batch * BATCH_POINTS * 7 * 7
        entry["tensor_core_spread_useful_tflops"] = useful / (spread_ms / 1e3) / 1e12 if spread_ms else None
        result[f"B{batch}"] = entry
        del c, out
        torch.cuda.empty_cache()
    return result


def radial_3d_line(w, torch, timed, barrier, world, dev, args, rank):
    """The 3D configuration: 256^3 modes, 4096 radial spokes x 12207 samples
    (49,999,872 points), eps 1e-5. Type-1 and type-2 NU points/s on prepared
    points with stage times, and rel-l2 against FP64 direct sums on 4 modes
    (type 1) and 64 points (type 2)."""
    from wgpunufft_b200 import workloads

    modes, count, eps, dist = workloads.CASES["radial"]
    pts = workloads.points(dist, count, 3, seed=SEED % 1000 + 31, device=dev)
    c = workloads.values(1, count, seed=SEED % 1000 + 32, device=dev)
    n = modes[0] * modes[1] * modes[2]
    result = {"workload": "3d_type1_type2_modes256^3_M49999872_radial_eps1e-5", "modes": list(modes),
              "points": count, "eps": eps, "unit": UNIT}
    steps = max(1, min(args.steps, 5))
    pts_h = pts.cpu().numpy().astype(np.float64) if rank == 0 else None
    plan = w.NufftPlan.type1_gpu(w.NufftConfig(modes, eps))
    plan.set_points_gpu(pts)
    out = torch.empty((1, n), dtype=torch.complex64, device=dev)
    for _ in range(max(1, args.warmup)):
        plan.execute_gpu_batch(1, c, out)
    barrier()
    plan.stage_timing(True)
    plan.stage_report()
    total = timed(lambda: plan.execute_gpu_batch(1, c, out), steps)
    stages = plan.stage_report()
    plan.stage_timing(False)
    (total,) = max_over_ranks([total], dev)
    item = {"value": replica_throughput(world, count, total, steps), "ms_per_step": total / steps,
            "stages_ms_per_step": {k: v[0] / steps for k, v in stages.items()}}
    if rank == 0:
        from oracle import native

        select = np.random.default_rng(9).choice(n, 4, replace=False)
        ref = native.direct_type1(pts_h, c.cpu().numpy().astype(np.complex128), modes, select=select)
        got = out.cpu().numpy()[:, select]
        item["rel_l2"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    result["type1"] = item
    del plan, out
    plan2 = w.NufftPlan.type2_gpu(w.NufftConfig(modes, eps))
    plan2.set_points_gpu(pts)
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 33)
    f = torch.complex(torch.randn((1, n), generator=g, device=dev), torch.randn((1, n), generator=g, device=dev))
    vals = torch.empty((1, count), dtype=torch.complex64, device=dev)
    for _ in range(max(1, args.warmup)):
        plan2.execute_gpu_batch(1, f, vals)
    barrier()
    total2 = timed(lambda: plan2.execute_gpu_batch(1, f, vals), steps)
    (total2,) = max_over_ranks([total2], dev)
    item2 = {"value": replica_throughput(world, count, total2, steps), "ms_per_step": total2 / steps}
    if rank == 0:
        from oracle import native

        pick = np.random.default_rng(10).choice(count, 64, replace=False)
        ref2 = native.direct_type2(pts_h[pick], f.cpu().numpy().astype(np.complex128), modes)
        got2 = vals.cpu().numpy()[:, pick]
        item2["rel_l2"] = float(np.linalg.norm(got2 - ref2) / np.linalg.norm(ref2))
    result["type2"] = item2
    del plan2, f, vals, pts, c
    torch.cuda.empty_cache()
    return result


def f64_line(w, torch, timed, barrier, world, dev, args, rank):
    """f64 plans of the batched configuration: 2D 512^2 modes, 2e6 uniform
    points, eps 1e-9 (w = 10) and 1e-12 (w = 13), one vector; type-1 and
    type-2 NU points/s with rel-l2 against FP64 direct sums (8 modes, 64
    points)."""
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 41)
    pts = (torch.rand((BATCH_POINTS, 2), generator=g, device=dev, dtype=torch.float64) * (2 * np.pi) - np.pi).contiguous()
    n = BATCH_MODES[0] * BATCH_MODES[1]
    steps = max(1, min(args.steps, 5))
    pts_h = pts.cpu().numpy() if rank == 0 else None
    result = {"workload": "2d_modes512x512_M2e6_uniform_f64", "modes": list(BATCH_MODES), "points": BATCH_POINTS,
              "unit": UNIT}
    for eps in (1e-9, 1e-12):
        entry = {}
        c = torch.complex(torch.randn((1, BATCH_POINTS), generator=g, device=dev, dtype=torch.float64),
                          torch.randn((1, BATCH_POINTS), generator=g, device=dev, dtype=torch.float64))
        f = torch.complex(torch.randn((1, n), generator=g, device=dev, dtype=torch.float64),
                          torch.randn((1, n), generator=g, device=dev, dtype=torch.float64))
        for kind in (1, 2):
            config = w.NufftConfig(BATCH_MODES, eps, precision=w.Precision.F64)
            plan = (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(config)
            plan.set_points_gpu(pts)
            inputs = c if kind == 1 else f
            out = torch.empty((1, n if kind == 1 else BATCH_POINTS), dtype=torch.complex128, device=dev)
            for _ in range(max(1, args.warmup)):
                plan.execute_gpu_batch(1, inputs, out)
            barrier()
            total = timed(lambda: plan.execute_gpu_batch(1, inputs, out), steps)
            (total,) = max_over_ranks([total], dev)
            item = {"value": replica_throughput(world, BATCH_POINTS, total, steps), "ms_per_step": total / steps,
                    "kernel_width": plan.kernel_width()}
            if rank == 0:
                from oracle import native

                if kind == 1:
                    select = np.random.default_rng(12).choice(n, 8, replace=False)
                    ref = native.direct_type1(pts_h, c.cpu().numpy(), BATCH_MODES, select=select)
                    got = out.cpu().numpy()[:, select]
                else:
                    pick = np.random.default_rng(13).choice(BATCH_POINTS, 64, replace=False)
                    ref = native.direct_type2(pts_h[pick], f.cpu().numpy(), BATCH_MODES)
                    got = out.cpu().numpy()[:, pick]
                item["rel_l2"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
            entry[f"type{kind}"] = item
            del plan, out
        result[f"eps{eps:g}"] = entry
    return result


def type3_line(w, torch, timed, barrier, world, dev, args, rank):
    """The 3D type-3 configuration: f64, 10^6 sources uniform in [-1, 1]^3 to
    10^6 targets uniform in [-200, 200]^3, eps 1e-9. Execution on set points
    (pre-phase, outer spread, inner type 2, post-phase) and set_points +
    execution, with rel-l2 against FP64 direct sums on 64 targets."""
    count = 1_000_000
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 51)
    src = (torch.rand((count, 3), generator=g, device=dev, dtype=torch.float64) * 2 - 1).contiguous()
    tgt = (torch.rand((count, 3), generator=g, device=dev, dtype=torch.float64) * 400 - 200).contiguous()
    c = torch.complex(torch.randn((1, count), generator=g, device=dev, dtype=torch.float64),
                      torch.randn((1, count), generator=g, device=dev, dtype=torch.float64))
    config = w.NufftType3Config(((-1.0, 1.0),) * 3, ((-200.0, 200.0),) * 3, eps=1e-9)
    plan = w.NufftType3Plan(config)
    out = torch.empty((1, count), dtype=torch.complex128, device=dev)
    steps = max(1, min(args.steps, 3))
    plan.set_points_gpu(src, tgt)
    for _ in range(max(1, args.warmup)):
        plan.execute_gpu_batch(1, c, out)
    barrier()
    total = timed(lambda: plan.execute_gpu_batch(1, c, out), steps)
    total_all = timed(lambda: plan.encode_gpu_batch(1, src, c, tgt, out), steps)
    (total, total_all) = max_over_ranks([total, total_all], dev)
    result = {"workload": "3d_type3_f64_src1e6_in[-1,1]^3_tgt1e6_in[-200,200]^3_eps1e-9", "unit": UNIT,
              "value": replica_throughput(world, count, total, steps), "ms_per_step": total / steps,
              "with_set_points": {"value": replica_throughput(world, count, total_all, steps),
                                  "ms_per_step": total_all / steps},
              "note": "points/s counts sources (= targets)"}
    if rank == 0:
        from oracle import native

        pick = np.random.default_rng(14).choice(count, 64, replace=False)
        ref = native.direct_type3(src.cpu().numpy(), c.cpu().numpy(), tgt.cpu().numpy()[pick], 1)
        got = out.cpu().numpy()[:, pick]
        result["rel_l2"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    del plan, out, src, tgt, c
    torch.cuda.empty_cache()
    result["small_outer_grids_f32"] = type3_small_grid_lines(w, torch, timed, barrier, world, dev, args, rank)
    return result


def type3_small_grid_lines(w, torch, timed, barrier, world, dev, args, rank):
    """Type 3 in f32 on small outer grids, the regime the reference serves with
    its dense small-grid spreader (src/gpu_dense_spread.rs:68-78: one or two
    axes, at most 2^16 cells): 10^6 sources uniform in [-1, 1]^d to 10^6
    targets uniform in [-30, 30]^d, eps 1e-6, d = 1 and 2. Here the binned
    spreader serves it, its parts sized so that every SM has work."""
    lines = {}
    count = 1_000_000
    steps = max(1, min(args.steps, 3))
    for d in (1, 2):
        g = torch.Generator(device=dev)
        g.manual_seed(SEED + 60 + d)
        src = (torch.rand((count, d), generator=g, device=dev) * 2 - 1).contiguous()
        tgt = (torch.rand((count, d), generator=g, device=dev) * 60 - 30).contiguous()
        c = torch.complex(torch.randn((1, count), generator=g, device=dev),
                          torch.randn((1, count), generator=g, device=dev))
        config = w.NufftType3Config(((-1.0, 1.0),) * d, ((-30.0, 30.0),) * d, eps=1e-6,
                                    precision=w.Precision.F32)
        plan = w.NufftType3Plan(config)
        out = torch.empty((1, count), dtype=torch.complex64, device=dev)
        plan.set_points_gpu(src, tgt)
        for _ in range(max(1, args.warmup)):
            plan.execute_gpu_batch(1, c, out)
        barrier()
        total = timed(lambda: plan.execute_gpu_batch(1, c, out), steps)
        (total,) = max_over_ranks([total], dev)
        line = {"workload": f"{d}d_type3_f32_src1e6_in[-1,1]^{d}_tgt1e6_in[-30,30]^{d}_eps1e-6", "unit": UNIT,
                "value": replica_throughput(world, count, total, steps), "ms_per_step": total / steps,
                "outer_grid": list(plan.info().outer_shape[:d])}
        if rank == 0:
            from oracle import native

            pick = np.random.default_rng(15 + d).choice(count, 64, replace=False)
            ref = native.direct_type3(src.double().cpu().numpy(), c.cpu().numpy().astype(np.complex128),
                                      tgt.double().cpu().numpy()[pick], 1)
            got = out.cpu().numpy()[:, pick]
            line["rel_l2"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        lines[f"{d}d"] = line
        del plan, out, src, tgt, c
    torch.cuda.empty_cache()
    return lines


def uneven_problems_line(w, torch, barrier, world, dev, args, rank):
    """256 independent type-1 problems of uneven sizes (2D/3D, 64^2..256^2 and
    32^3..64^3 modes, 1e3..1e6 points, uniform or clustered, eps 1e-6), one
    plan each with its points set: all executions issued one after another
    (eager) and replayed from one captured CUDA graph."""
    from wgpunufft_b200 import workloads

    problems = workloads.uneven_problems(256, seed=SEED % 1000)
    stream = torch.cuda.Stream()
    plans, outs = [], []
    with torch.cuda.stream(stream):
        for modes, p, c in problems:
            plan = w.NufftPlan.type1_gpu(w.NufftConfig(modes, 1e-6))
            plan.set_points_gpu(p, stream=stream)
            out = torch.empty((1, int(np.prod(modes))), dtype=torch.complex64, device=dev)
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

        def timed_on(fn, steps):
            total = 0.0
            for _ in range(steps):
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(stream)
                fn()
                end.record(stream)
                end.synchronize()
                total += start.elapsed_time(end)
            return total

        steps = max(1, min(args.steps, 5))
        for _ in range(2):
            run_all()
            graph.replay()
        barrier()
        eager_ms = timed_on(run_all, steps)
        graph_ms = timed_on(graph.replay, steps)
    del graph
    eager_ms, graph_ms = max_over_ranks([eager_ms, graph_ms], dev)
    total_points = sum(int(p.shape[0]) for _, p, _ in problems)
    return {"problems": len(problems), "points": total_points, "eps": 1e-6,
            "graph": {"value": replica_throughput(world, total_points, graph_ms, steps), "unit": UNIT,
                      "ms_per_step": graph_ms / steps},
            "eager": {"value": replica_throughput(world, total_points, eager_ms, steps), "unit": UNIT,
                      "ms_per_step": eager_ms / steps},
            "note": "one plan per problem (prepared points); a step executes all 256"}


def profile_traffic():
    """DRAM bytes per spread launch from the committed ncu summary, if present."""
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

    dev = f"cuda:{local}"
    points_h, strengths_h = make_inputs()
    points = torch.from_numpy(points_h).to(dev)
    strengths = torch.from_numpy(strengths_h.view(np.float32)).to(dev).view(torch.complex64)
    config = w.NufftConfig(MODES, EPS)
    plan = w.NufftPlan.type1_gpu(config, device=local)
    out = torch.empty(config.mode_count(), dtype=torch.complex64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(step_fn, steps):
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(float(i))
            starts[i].record(stream)
            step_fn()
            ends[i].record(stream)
        torch.cuda.synchronize()
        return sum(s.elapsed_time(e) for s, e in zip(starts, ends))

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
    barrier()
    with ClockSampler(local) as clocks:
        total_ms = timed(lambda: plan.execute_type1_gpu(strengths, out), args.steps)
        launches = w.launch_count() - launches0
        stages = plan.stage_report()
        plan.stage_timing(False)
        one_shot_ms = timed(lambda: plan.encode_type1_gpu(points, strengths, out), args.steps)
    barrier()
    clock_summary = clocks.summary()
    total_ms, one_shot_ms = max_over_ranks([total_ms, one_shot_ms], dev)
    ms = total_ms / args.steps
    value = replica_throughput(world, POINTS, total_ms, args.steps)
    one_shot = replica_throughput(world, POINTS, one_shot_ms, args.steps)

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
    type2_ms = timed(lambda: plan2.execute_type2_gpu(coefficients, values), args.steps)
    stages2 = plan2.stage_report()
    plan2.stage_timing(False)
    type2_one_shot_ms = timed(lambda: plan2.encode_type2_gpu(points, coefficients, values), args.steps)
    type2_ms, type2_one_shot_ms = max_over_ranks([type2_ms, type2_one_shot_ms], dev)
    type2 = {"value": replica_throughput(world, POINTS, type2_ms, args.steps), "unit": UNIT,
             "ms_per_step": type2_ms / args.steps,
             "one_shot_value": replica_throughput(world, POINTS, type2_one_shot_ms, args.steps),
             "stages_ms_per_step": {k: v[0] / args.steps for k, v in stages2.items()}}

    # Accuracy of this output against FP64 direct sums on 16 seeded modes.
    rel = None
    if rank == 0:
        from oracle import native

        plan.execute_type1_gpu(strengths, out)
        plan.synchronize()
        got = out.cpu().numpy()
        select = np.random.default_rng(1).choice(config.mode_count(), 16, replace=False)
        ref = native.direct_type1(points_h.astype(np.float64), strengths_h, MODES, select=select)[0]
        rel = float(np.linalg.norm(got[select] - ref) / np.linalg.norm(ref))

    # End to end through the reference-facing C interface with host buffers:
    # wgpu_nufftf_setpts (per-axis f32 coordinates) + wgpu_nufftf_execute
    # every step, as a Fortran/MATLAB/Julia caller of the reference would.
    e2e = None
    if not args.no_e2e:
        e2e = c_interface_e2e(w, torch, points_h, strengths_h, timed, barrier, world, dev, args)

    # Batched vectors on one point set (2D 512^2 modes, 2e6 points, eps 1e-6):
    # the tensor-core spreader against the CUDA-core spreader on the same plan
    # shape and inputs.
    batched = None
    if not args.no_batched:
        batched = batched_comparison(w, torch, timed, barrier, world, dev, args, rank)
    uneven = None
    if not args.no_uneven:
        uneven = uneven_problems_line(w, torch, barrier, world, dev, args, rank)
    # The 3D radial configuration (256^3 modes, 5e7 points, eps 1e-5).
    radial = None
    if not args.no_radial:
        radial = radial_3d_line(w, torch, timed, barrier, world, dev, args, rank)
    # f64 plans (2D 512^2 modes, 2e6 points, eps 1e-9 and 1e-12).
    f64 = None
    if not args.no_f64:
        f64 = f64_line(w, torch, timed, barrier, world, dev, args, rank)
    # The 3D type-3 f64 configuration (10^6 sources to 10^6 targets).
    type3 = None
    if not args.no_type3:
        type3 = type3_line(w, torch, timed, barrier, world, dev, args, rank)

    if rank == 0:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
        hbm = peaks.get("hbm_gbs", 6650.0)
        spread_ms, spread_launches = stages.get("spread", (0.0, 0))
        per_launch_ms = spread_ms / max(spread_launches, 1)
        fine = plan.fine_grid_shape()
        algorithmic = POINTS * (4 * 2 + 8 + 4) + fine[0] * fine[1] * 8
        achieved = algorithmic / (per_launch_ms / 1e3) / 1e9 if per_launch_ms > 0 else None
        roofline = {"bound": "hbm", "kernel": "spread_tiles_kernel<2,6>", "achieved": achieved, "peak": hbm,
                    "unit": "GB/s", "frac": achieved / hbm if achieved else None,
                    "traffic": profile_traffic(),
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650 GB/s",
                    "algorithmic_bytes_per_launch": algorithmic}
        cpu = None
        if not args.no_cpu:
            sample_pts, sample_str = points_h[:CPU_SAMPLE], strengths_h[:CPU_SAMPLE]
            cpu_value, threads, cpu_s = cpu_plan_throughput(sample_pts, sample_str)
            cpu = {"value": cpu_value, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"first {CPU_SAMPLE:,} of the {POINTS:,} points, same plan; restated CpuNufftPlan one-shot execute, median of 3 ({cpu_s:.2f} s each)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded uniform points, N(0,1) strengths)",
            "config": {"workload": WORKLOAD, "modes": list(MODES), "points": POINTS, "eps": EPS, "batch": 1,
                       "fine_grid": list(fine), "kernel_width": plan.kernel_width(),
                       "l2": "flushed between steps by a 256 MiB write outside the timed events",
                       "parallelism": f"replicas x{world}"},
            "one_shot": {"value": one_shot, "unit": UNIT, "ms_per_step": one_shot_ms / args.steps,
                         "note": "set_points (stable bin sort) + execute per step"},
            "rel_l2": rel,
            "stages_ms_per_step": {k: v[0] / args.steps for k, v in stages.items()},
            "type2": type2,
            "batched": batched,
            "uneven_problems": uneven,
            "radial_3d": radial,
            "f64": f64,
            "type3": type3,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clock_summary,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
