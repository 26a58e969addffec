"""Autotuner of the spreader's launch choices, run on a B200:

    python -m wgpunufft_b200.tune [--out PATH] [--repeats N] [--tensor-only]

For every workload below (the benchmark configurations and the sizes of the
uneven-problems batch), it measures type-1 executions on prepared points
under every candidate choice (tile side, CTAs per SM the tile parts are
sized for, the same on crowded one-cell bins) and, for batched workloads,
the smallest batch at which the tensor cores beat the CUDA cores, per
plan type and window width (eps 1e-3 and 1e-6); then it writes the fastest
choice per workload key (plan type, dimension, precision, window width,
log2 fine-grid cells, log2 points per cell) as tuning_table.h.
`--tensor-only` measures the tensor-core thresholds alone and merges them
into the table already written. The library compiles that table in, so a key always gets
the same choices and outputs stay bitwise repeatable. Inputs are seeded
synthetic points (uniform, clustered, radial) and N(0, 1) strengths.
"""

from __future__ import annotations

import argparse
import itertools
import json
import math
import re
import statistics
from pathlib import Path

HERE = Path(__file__).resolve().parent

# (name, modes, points, eps, distribution, precision)
WORKLOADS = [
    ("2d_1024_1e7_uniform", (1024, 1024), 10_000_000, 1e-5, "uniform", "f32"),
    ("2d_1024_1e7_clustered", (1024, 1024), 10_000_000, 1e-5, "clustered", "f32"),
    ("2d_512_2e6_uniform", (512, 512), 2_000_000, 1e-6, "uniform", "f32"),
    ("2d_64_1e5_uniform", (64, 64), 100_000, 1e-6, "uniform", "f32"),
    ("2d_128_1e4_uniform", (128, 128), 10_000, 1e-6, "uniform", "f32"),
    ("2d_128_1e6_clustered", (128, 128), 1_000_000, 1e-6, "clustered", "f32"),
    ("2d_256_1e5_uniform", (256, 256), 100_000, 1e-6, "uniform", "f32"),
    ("3d_256_5e7_radial", (256, 256, 256), 4096 * 12207, 1e-5, "radial", "f32"),
    ("3d_64_1e6_uniform", (64, 64, 64), 1_000_000, 1e-6, "uniform", "f32"),
    ("3d_32_1e5_clustered", (32, 32, 32), 100_000, 1e-6, "clustered", "f32"),
    ("2d_512_2e6_f64_1e-9", (512, 512), 2_000_000, 1e-9, "uniform", "f64"),
]

CANDIDATES = {
    2: {"tile": (32, 64), "ctas_per_sm": (2, 4, 8), "crowded_ctas_per_sm": (1, 2)},
    3: {"tile": (8, 16), "ctas_per_sm": (2, 4), "crowded_ctas_per_sm": (1,)},
}
F64_CANDIDATES = {"tile": (16, 32), "ctas_per_sm": (2, 4, 8), "crowded_ctas_per_sm": (1,)}


def _points(torch, workloads, dist, count, d, dtype):
    p = workloads.points(dist, count, d, seed=11)
    return p.to(dtype).contiguous()


def _time(torch, fn, repeats):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(repeats):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        fn()
        end.record()
        end.synchronize()
        times.append(start.elapsed_time(end))
    return statistics.median(times)


def tune_workload(torch, w, workloads, native, spec, repeats):
    name, modes, count, eps, dist, precision = spec
    d = len(modes)
    f64 = precision == "f64"
    real = torch.float64 if f64 else torch.float32
    pts = _points(torch, workloads, dist, count, d, real)
    c = workloads.values(1, count, seed=12).to(torch.complex128 if f64 else torch.complex64)
    config = w.NufftConfig(modes, eps, precision=w.Precision.F64 if f64 else w.Precision.F32)
    out = torch.empty((1, config.mode_count()), dtype=c.dtype, device="cuda")
    grid = F64_CANDIDATES if f64 else CANDIDATES[d]
    results = []
    for tile, ctas, crowded in itertools.product(grid["tile"], grid["ctas_per_sm"], grid["crowded_ctas_per_sm"]):
        t = native.Tuning(tile, ctas, crowded, 0)
        native.library().b200nufft_tuning_override(t)
        plan = w.NufftPlan.type1_gpu(config)
        plan.set_points_gpu(pts)
        ms = _time(torch, lambda: plan.execute_gpu_batch(1, c, out), repeats)
        results.append({"tile": tile, "ctas_per_sm": ctas, "crowded_ctas_per_sm": crowded, "ms": ms})
        del plan
    native.library().b200nufft_tuning_override(None)
    plan = w.NufftPlan.type1_gpu(config)
    info = plan.info()
    fine_cells = math.prod(info.fine_shape[a] for a in range(d))
    best = min(results, key=lambda r: r["ms"])
    key = {"type": 1, "dimensions": d, "precision": 1 if f64 else 3, "width": info.kernel_width,
           "log2_cells": int(math.floor(math.log2(fine_cells))),
           "log2_density": max(-16, min(16, int(math.floor(math.log2(count / fine_cells)))))}
    del plan, pts, c, out
    torch.cuda.empty_cache()
    return {"workload": name, "key": key, "best": best, "candidates": results}


# The batched configuration the tensor-core thresholds are measured on (2D
# 512^2 modes, 2e6 uniform points), its window widths (eps) and batches.
TENSOR_MODES, TENSOR_POINTS = (512, 512), 2_000_000
TENSOR_EPS = (1e-2, 1e-3, 1e-4, 1e-5, 1e-6)
TENSOR_BATCHES = (16, 32, 64, 128, 256)


def tune_tensor_threshold(torch, w, workloads, native, kind, eps, repeats):
    """Smallest batch of TENSOR_BATCHES at which the tensor cores are faster
    on the batched configuration at `eps` (0 for none), the window width and
    the times per batch."""
    modes, count = TENSOR_MODES, TENSOR_POINTS
    pts = workloads.points("uniform", count, 2, seed=13)
    n = modes[0] * modes[1]
    times = {}
    width = 0
    for batch in TENSOR_BATCHES:
        inputs = workloads.values(batch, count if kind == 1 else n, seed=14)
        out = torch.empty((batch, n if kind == 1 else count), dtype=torch.complex64, device="cuda")
        ms = {}
        for method in (w.SpreadMethod.TENSOR_CORES, w.SpreadMethod.CUDA_CORES):
            plan = (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(
                w.NufftConfig(modes, eps, batch=batch, spread_method=method))
            width = plan.kernel_width()
            plan.set_points_gpu(pts)
            ms[method] = _time(torch, lambda: plan.execute_gpu_batch(batch, inputs, out), repeats)
            del plan
        del inputs, out
        torch.cuda.empty_cache()
        times[batch] = {"tensor_cores": ms[w.SpreadMethod.TENSOR_CORES], "cuda_cores": ms[w.SpreadMethod.CUDA_CORES]}
        if ms[w.SpreadMethod.TENSOR_CORES] < ms[w.SpreadMethod.CUDA_CORES]:
            return batch, width, times
    return 0, width, times


def nearest(entries, key):
    """The entry the library's lookup (csrc/tuning.cpp tuning_for) gives a
    key: same type, dimensions, precision and width, least 4 |log2 cells
    difference| + |log2 density difference|, the first on ties; None."""
    best, best_distance = None, None
    for e in entries:
        k = e["key"]
        if any(k[f] != key[f] for f in ("type", "dimensions", "precision", "width")):
            continue
        distance = 4 * abs(k["log2_cells"] - key["log2_cells"]) + abs(k["log2_density"] - key["log2_density"])
        if best_distance is None or distance < best_distance:
            best, best_distance = e, distance
    return best


def tensor_entries(torch, w, workloads, native, entries, repeats):
    """Sets the tensor-core threshold of every (type, width) of the batched
    configuration's key: the tuned entry's where the key exists, else a new
    entry with the plan's default launch choices. Returns the measurements."""
    modes, count = TENSOR_MODES, TENSOR_POINTS
    fine_cells = 4 * modes[0] * modes[1]
    cells = int(math.floor(math.log2(fine_cells)))
    density = max(-16, min(16, int(math.floor(math.log2(count / fine_cells)))))
    measured = []
    for kind in (1, 2):
        for eps in TENSOR_EPS:
            threshold, width, times = tune_tensor_threshold(torch, w, workloads, native, kind, eps, repeats)
            measured.append({"type": kind, "eps": eps, "width": width, "threshold": threshold, "ms": times})
            print(json.dumps(measured[-1]), flush=True)
            key = {"type": kind, "dimensions": 2, "precision": 3, "width": width, "log2_cells": cells,
                   "log2_density": density}
            value = threshold or 1 << 30
            found = False
            for e in entries:
                if e["key"] == key:
                    e["tensor_min_batch"] = value
                    found = True
            if not found:
                # The launch choices the key got before it had an entry (the
                # nearest type-1 entry of its width, as the library looks it
                # up; they do not apply to interpolation), else the plan's
                # defaults; the time noted is the CUDA cores' on the
                # smallest batch.
                source = nearest(entries, dict(key, type=1))
                best = dict(source["best"]) if source else {"tile": 0, "ctas_per_sm": 4, "crowded_ctas_per_sm": 1}
                first = TENSOR_BATCHES[0]
                best["ms"] = times[first]["cuda_cores"]
                name = f"2d_512_2e6_uniform_eps{eps:g}_type{kind}_cuda_cores_B{first}"
                entries.append({"workload": name, "key": key, "best": best, "tensor_min_batch": value})
    return measured


ENTRY = re.compile(r"^\s*\{([-\d, ]+)\},\s*// (\S+): ([\d.]+) ms")


def read_table(path):
    """The entries of a tuning_table.h written by table_header."""
    entries = []
    for line in Path(path).read_text().splitlines():
        m = ENTRY.match(line)
        if not m:
            continue
        v = [int(x) for x in m.group(1).split(",")]
        key = dict(zip(("type", "dimensions", "precision", "width", "log2_cells", "log2_density"), v[:6]))
        best = {"tile": v[6], "ctas_per_sm": v[7], "crowded_ctas_per_sm": v[8], "ms": float(m.group(3))}
        entries.append({"workload": m.group(2), "key": key, "best": best, "tensor_min_batch": v[9]})
    return entries


def merge_keys(entries):
    """One entry per key: workloads of the same key (uniform and clustered
    points of one size and density) take the candidate with the least total
    time over all of them."""
    merged = {}
    for e in entries:
        k = tuple(sorted(e["key"].items()))
        merged.setdefault(k, []).append(e)
    out = []
    for group in merged.values():
        if len(group) == 1 or not all(g.get("candidates") for g in group):
            out.append(group[0])
            continue
        totals = {}
        for g in group:
            for c in g["candidates"]:
                choice = (c["tile"], c["ctas_per_sm"], c["crowded_ctas_per_sm"])
                totals[choice] = totals.get(choice, 0.0) + c["ms"]
        choice = min(totals, key=totals.get)
        best = {"tile": choice[0], "ctas_per_sm": choice[1], "crowded_ctas_per_sm": choice[2], "ms": totals[choice]}
        names = "+".join(g["workload"] for g in group)
        out.append(dict(group[0], workload=names, best=best))
    return out


def table_header(entries):
    lines = ["// Tuned launch choices per workload key, written by wgpunufft_b200/tune.py",
             "// from measurements on a B200. Fields: type, dimensions, precision, width,",
             "// log2 fine-grid cells, log2 density; tile side, CTAs per SM, CTAs per SM",
             "// on crowded one-cell bins, smallest tensor-core batch.",
             "#pragma once", "", "namespace b200nufft {", "",
             "struct TuningEntry {",
             "  int type, dimensions, precision, width, log2_cells, log2_density;",
             "  int tile, ctas_per_sm, crowded_ctas_per_sm, tensor_min_batch;",
             "};", "", "constexpr TuningEntry kTuningTable[] = {"]
    for e in entries:
        k, b = e["key"], e["best"]
        lines.append(f"    {{{k['type']}, {k['dimensions']}, {k['precision']}, {k['width']}, {k['log2_cells']}, "
                     f"{k['log2_density']}, {b['tile']}, {b['ctas_per_sm']}, {b['crowded_ctas_per_sm']}, "
                     f"{e.get('tensor_min_batch', 16)}}},  // {e['workload']}: {b['ms']:.4f} ms")
    lines += ["};", f"constexpr int kTuningEntries = {len(entries)};", "", "}  // namespace b200nufft", ""]
    return "\n".join(lines)


def main():
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("--out", default=str(HERE / "csrc" / "tuning_table.h"))
    parser.add_argument("--report", default=None, help="JSON file for every measurement")
    parser.add_argument("--from-report", default=None, help="write the table from an earlier report, no GPU")
    parser.add_argument("--repeats", type=int, default=5)
    parser.add_argument("--tensor-only", action="store_true",
                        help="measure the tensor-core thresholds alone and merge them into --out")
    args = parser.parse_args()
    if args.from_report:
        entries = json.loads(Path(args.from_report).read_text())["entries"]
        Path(args.out).write_text(table_header(merge_keys(entries)))
        return
    import torch

    import wgpunufft_b200 as w
    from wgpunufft_b200 import _native as native
    from wgpunufft_b200 import workloads

    if args.tensor_only:
        entries = read_table(args.out)
    else:
        entries = []
        for spec in WORKLOADS:
            entry = tune_workload(torch, w, workloads, native, spec, args.repeats)
            entries.append(entry)
            print(json.dumps({"workload": entry["workload"], "best": entry["best"]}), flush=True)
        entries = merge_keys(entries)
    measured = tensor_entries(torch, w, workloads, native, entries, args.repeats)
    Path(args.out).write_text(table_header(entries))
    report = {"entries": entries, "tensor_thresholds": measured}
    if args.report:
        Path(args.report).write_text(json.dumps(report, indent=1))
    print(json.dumps({"written": args.out, "tensor_thresholds": [(m["type"], m["width"], m["threshold"])
                                                                  for m in measured]}), flush=True)


if __name__ == "__main__":
    main()
