"""Spreader layout and bin-geometry choice restated from src/gpu_nd_spread.rs:194-459
(oracle; test infrastructure). Precision is "F32", "F64" or "Df64"; device
limits are wgpu's defaults (256 invocations per workgroup)."""

from __future__ import annotations

import math

MAX_BLOCK_EDGE = 16
MAX_ROW_BATCH = 128
MAX_ROWS = 1 << 20
TARGET_REACH_ROWS = 1024.0
MAX_BINS = 1 << 23
MAX_COARSENING = 3
BATCH_COST = 100.0
ROW_COST = 1.0
BIN_COST = 0.1
COST_TOLERANCE = 0.1
MAX_INVOCATIONS = 256


def _div_ceil(a: int, b: int) -> int:
    return -(-a // b)


def _next_pow2(v: int) -> int:
    p = 1
    while p < v:
        p <<= 1
    return p


def target_workgroup_size(d: int, precision: str) -> int:
    if d == 1:
        return 64
    if d == 2 and precision == "F32":
        return 32
    if (d in (2, 3) and precision == "F64") or precision == "F32":
        return 64
    return 256


def max_run(d: int, precision: str) -> int:
    if d == 1 or (d == 2 and precision == "Df64"):
        return 2
    if d == 2:
        return 4
    if d == 3 or precision in ("F64", "Df64"):
        return 8
    return 16


def segment_length(max_parts: int) -> int:
    """segment_length (src/gpu_nd_spread.rs:598-601)."""
    bit = max(max_parts, 1).bit_length() - 1
    return 1 << ((bit + 1) // 2)


class Geometry:
    def __init__(self, side, bins, full, reach_bins, mean_reach_bins):
        self.side = side
        self.bins = bins
        self.full = full
        self.reach_bins = reach_bins
        self.mean_reach_bins = mean_reach_bins

    def bin_count(self) -> int:
        return math.prod(self.bins)

    def rows(self) -> int:
        return max(math.prod(self.reach_bins[1:]), 1)


class Layout:
    """NdSpreadLayout::for_grid and choose_geometry."""

    def __init__(self, width: int, fine_shape, precision: str = "F32"):
        fine = list(fine_shape)
        d = len(fine)
        self.width = width
        self.fine_shape = fine
        target = max(min(target_workgroup_size(d, precision), MAX_INVOCATIONS), 1)

        def edge_limit(axis):
            return max(fine[axis] + 1 - width, 1)

        run_cap = min(max_run(d, precision), edge_limit(0))
        run = 1
        while run * 2 <= run_cap:
            run *= 2
        block = [1] * d
        invocations = 1
        while True:
            candidates = [a for a in range(1, d)
                          if block[a] * 2 <= min(edge_limit(a), MAX_BLOCK_EDGE) and invocations * 2 <= target]
            if not candidates:
                break
            # min_by_key keeps the first minimum of (block, usize::MAX - n).
            axis = min(candidates, key=lambda a: (block[a], -fine[a]))
            block[axis] *= 2
            invocations *= 2
        groups_0 = 1
        while invocations * 2 <= target and run * groups_0 * 2 <= edge_limit(0):
            groups_0 *= 2
            invocations *= 2
        block[0] = run * groups_0
        workgroup_size = groups_0 * math.prod(block[1:])

        def reach_cells(axis):
            return block[axis] + width - 1

        side = [1] * d
        if d != 2 or precision != "F32":
            side[0] = 2

        def mean_reach(sides, axis):
            return min((reach_cells(axis) - 1) / sides[axis] + 1.0, float(_div_ceil(fine[axis], sides[axis])))

        while True:
            rows = math.prod(mean_reach(side, a) for a in range(1, d)) if d > 1 else 1.0
            bin_count = math.prod(_div_ceil(fine[a], side[a]) for a in range(d))
            if rows <= TARGET_REACH_ROWS and bin_count <= MAX_BINS:
                break
            widest = None
            for a in range(1, d):
                if side[a] < fine[a] and (widest is None or not (mean_reach(side, a) < mean_reach(side, widest))):
                    widest = a  # max_by keeps the last maximum
            if widest is not None:
                axis = widest
            elif bin_count > MAX_BINS and side[0] < fine[0]:
                axis = 0
            else:
                break
            side[axis] *= 2

        def geometry(sides):
            bins, full, reach, mean = [], [], [], []
            for a in range(d):
                count = _div_ceil(fine[a], sides[a])
                whole = reach_cells(a) + sides[a] > fine[a]
                bins.append(count)
                full.append(whole)
                reach.append(count if whole else min(count, _div_ceil(reach_cells(a), sides[a]) + 2))
                mean.append(mean_reach(sides, a))
            return Geometry(list(sides), bins, full, reach, mean)

        finest = geometry(side)
        while math.prod(finest.reach_bins[1:]) > MAX_ROWS:
            axes = [a for a in range(1, d) if finest.reach_bins[a] > 1]
            if not axes:
                break
            axis = max(axes, key=lambda a: (finest.reach_bins[a], a))  # last maximum
            side[axis] *= 2
            finest = geometry(side)
        geometries = [finest]
        for others in range(1, MAX_COARSENING + 1):
            for first in range(others + 1):
                sides = [min(side[a] << (first if a == 0 else others), _next_pow2(fine[a])) for a in range(d)]
                if all(g.side != sides for g in geometries):
                    geometries.append(geometry(sides))
        rows = geometries[0].rows()
        self.run = run
        self.groups_0 = groups_0
        self.block = block
        self.blocks = [_div_ceil(fine[a], block[a]) for a in range(d)]
        self.geometries = geometries
        self.workgroup_size = workgroup_size
        self.row_batch = max(min(MAX_ROW_BATCH, workgroup_size, _next_pow2(rows)), 1)

    def block_cells(self) -> int:
        return self.workgroup_size * self.run

    def choose_geometry(self, point_count: int) -> int:
        fine = self.fine_shape
        d = len(fine)
        density = point_count / math.prod(fine)
        blocks = float(math.prod(self.blocks))
        record_cost = self.workgroup_size * (d + 1.0) ** 2 / 1024.0
        estimates = []
        for g in self.geometries:
            rows = math.prod(g.mean_reach_bins[1:]) if d > 1 else 1.0
            batches = math.ceil(rows / self.row_batch)
            staged = math.prod(min(g.mean_reach_bins[a] * g.side[a], float(fine[a])) for a in range(d))
            cost = blocks * (BATCH_COST * batches + ROW_COST * rows + record_cost * density * staged) \
                + BIN_COST * g.bin_count()
            estimates.append((staged, cost))
        least = min(c for _, c in estimates)
        best = None
        for index, (staged, cost) in enumerate(estimates):
            if cost <= least * (1.0 + COST_TOLERANCE) and (best is None or staged < estimates[best][0]):
                best = index
        return 0 if best is None else best
