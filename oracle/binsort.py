"""Stable type-1 binning and type-2 grouped bins in numpy float32 (oracle; test infrastructure).

Restates the count / scatter / sort / prepare passes of src/gpu_nd_bins.rs:336-709
as their net effect - points sorted by bin key with ties in original index
order, the exclusive scan of the bin counts with a trailing total, and the
prepared slots - with the position fold of src/gpu_nd_wgsl.rs:198-298 written
as the double-float (df64) sequence of float32 operations that the CUDA
kernels execute: Knuth two-sum, Dekker split and two-product, quick-two-sum
renormalisation, no fused multiply-add.
"""

from __future__ import annotations

import math

import numpy as np

F = np.float32
FOLD_REACH_BITS = np.uint32(0x41490FDB)  # bits of 4*pi as f32


def _two_sum(a, b):
    s = (a + b).astype(F)
    v = (s - a).astype(F)
    e = ((a - (s - v)).astype(F) + (b - v).astype(F)).astype(F)
    return s, e


def _quick_two_sum(a, b):
    s = (a + b).astype(F)
    e = (b - (s - a)).astype(F)
    return s, e


def df64_add(ah, al, bh, bl):
    sh, sl = _two_sum(ah, bh)
    e = ((sl + al).astype(F) + bl).astype(F)
    return _quick_two_sum(sh, e)


def df64_sub(ah, al, bh, bl):
    return df64_add(ah, al, (-bh).astype(F), (-bl).astype(F))


def _split(a):
    t = (F(4097.0) * a).astype(F)
    hi = (t - (t - a).astype(F)).astype(F)
    lo = (a - hi).astype(F)
    return hi, lo


def _two_prod(a, b):
    p = (a * b).astype(F)
    ah, al = _split(a)
    bh, bl = _split(b)
    e = ((((ah * bh).astype(F) - p).astype(F) + (ah * bl).astype(F)).astype(F) + (al * bh).astype(F)).astype(F)
    e = (e + (al * bl).astype(F)).astype(F)
    return p, e


def df64_mul(ah, al, bh, bl):
    ph, pl = _two_prod(ah, bh)
    cross = ((ah * bl).astype(F) + (al * bh).astype(F)).astype(F)
    e = (pl + cross).astype(F)
    return _quick_two_sum(ph, e)


class AxisFold:
    """Constants of one axis: scale n/(2 pi) as a (hi, lo) float pair, origin floor(n/2)."""

    def __init__(self, n: int):
        scale = n / (2.0 * math.pi)
        self.n = n
        self.scale_hi = F(scale)
        self.scale_lo = F(scale - float(self.scale_hi))
        self.origin = F(n // 2)
        self.length = F(n)


def fold_position(x, axis: AxisFold):
    """fold_position (src/gpu_nd_wgsl.rs:258-266): df64 position in [0, n)."""
    x = np.asarray(x, dtype=F)
    zero = np.zeros_like(x)
    mh, ml = df64_mul(x, zero, np.full_like(x, axis.scale_hi), np.full_like(x, axis.scale_lo))
    ph, pl = df64_add(mh, ml, np.full_like(x, axis.origin), zero)
    n = np.full_like(x, axis.length)
    for _ in range(2):
        neg = (ph < 0) | ((ph == 0) & (pl < 0))
        ah, al = df64_add(ph, pl, n, zero)
        ph, pl = np.where(neg, ah, ph), np.where(neg, al, pl)
    for _ in range(2):
        big = (ph > n) | ((ph == n) & (pl >= 0))
        sh, sl = df64_sub(ph, pl, n, zero)
        ph, pl = np.where(big, sh, ph), np.where(big, sl, pl)
    return ph, pl


def df64_ceil(h, l):
    """ceil_df64_to_i32 (src/gpu_nd_wgsl.rs:281-286)."""
    base = np.floor(h).astype(F)
    rh, rl = df64_sub(h, l, base, np.zeros_like(base))
    positive = (rh > 0) | ((rh == 0) & (rl > 0))
    return base.astype(np.int64) + positive.astype(np.int64)


def support(x, axis: AxisFold, width: int):
    """Support start ceil(position - w/2) and offset start - position as (hi, lo).
    Coordinates outside the fold's reach give unspecified values; callers mask them."""
    with np.errstate(invalid="ignore", over="ignore"):
        return _support(x, axis, width)


def _support(x, axis: AxisFold, width: int):
    ph, pl = fold_position(x, axis)
    hw = np.full_like(ph, F(0.5 * width))
    sh, sl = df64_sub(ph, pl, hw, np.zeros_like(ph))
    start = df64_ceil(sh, sl)
    oh, ol = df64_sub(start.astype(F), np.zeros_like(ph), ph, pl)
    return start, oh, ol


def in_reach(x):
    bits = np.asarray(x, dtype=F).view(np.uint32) & np.uint32(0x7FFFFFFF)
    return bits <= FOLD_REACH_BITS


def _ilog2(v: int) -> int:
    return int(v).bit_length() - 1


def type1_keys(points: np.ndarray, fine, width: int, sides):
    """Bin keys of src/gpu_nd_bins.rs:474-554: starts of all axes wrapped onto
    the grid when every coordinate is within the fold's reach, else zero."""
    points = np.asarray(points, dtype=F).reshape(-1, len(fine))
    reach = np.all(in_reach(points), axis=1)
    key = np.zeros(points.shape[0], dtype=np.int64)
    stride = 1
    for a, n in enumerate(fine):
        start, _, _ = support(points[:, a], AxisFold(n), width)
        start = np.where(reach, start, 0)
        wrapped = np.clip(np.where(start < 0, start + n, start), 0, n - 1)
        key += (wrapped >> _ilog2(sides[a])) * stride
        stride *= -(-n // sides[a])
    return key, stride


FOLD_REACH64 = 4.0 * math.pi


def support64(x, n: int, width: int):
    """The F64 fold of src/gpu_nd_wgsl.rs:311-365 in numpy float64 (separate
    multiply and add): support start and offset start - position."""
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(invalid="ignore", over="ignore"):
        position = x * (n / (2.0 * math.pi)) + float(n // 2)
        for _ in range(2):
            position = np.where(position < 0.0, position + n, position)
        for _ in range(2):
            position = np.where(position >= n, position - n, position)
        start = np.ceil(position - 0.5 * width)
        offset = start - position
    return start, offset


def type1_keys64(points: np.ndarray, fine, width: int, sides):
    """Support-start bin keys of f64 coordinates (native f64 fold)."""
    points = np.asarray(points, dtype=np.float64).reshape(-1, len(fine))
    reach = np.all(np.abs(points) <= FOLD_REACH64, axis=1)
    key = np.zeros(points.shape[0], dtype=np.int64)
    stride = 1
    for a, n in enumerate(fine):
        start, _ = support64(points[:, a], n, width)
        start = np.where(reach, start, 0).astype(np.int64)
        wrapped = np.clip(np.where(start < 0, start + n, start), 0, n - 1)
        key += (wrapped >> _ilog2(sides[a])) * stride
        stride *= -(-n // sides[a])
    return key, stride


def type2_sides64(fine):
    """type2_bin_shape (src/gpu_nd.rs:566-586): 4 cells per axis, doubled from
    the last axis backwards while there are more than 2^24 bins."""
    sides = [4] * len(fine)
    axis = len(fine)
    while math.prod(-(-n // s) for n, s in zip(fine, sides)) > (1 << 24):
        axis = len(fine) - 1 if axis == 0 else axis - 1
        sides[axis] *= 2
    return sides


def approximate_cell(x, axis: AxisFold):
    """approximate_cell (src/gpu_point_bins.rs:460-464) in plain f32."""
    x = np.asarray(x, dtype=F)
    position = ((x * axis.scale_hi).astype(F) + axis.origin).astype(F)
    with np.errstate(invalid="ignore", over="ignore"):
        q = np.floor((position / axis.length).astype(F)).astype(F)
        wrapped = (position - (axis.length * q).astype(F)).astype(F)
        clamped = np.fmax(wrapped, F(0))
        cell = np.where(clamped >= F(4294967040.0), np.float64(2**32 - 1), clamped).astype(np.float64)
    cell = np.floor(cell).astype(np.int64)
    return np.minimum(cell, axis.n - 1)


def type2_keys(points: np.ndarray, fine):
    """Type-2 grouped bin keys: sides 8 in 1D and 2D, 4 in 3D (src/gpu_2d.rs:22, src/gpu_3d.rs:25)."""
    d = len(fine)
    side = 4 if d == 3 else 8
    points = np.asarray(points, dtype=F).reshape(-1, d)
    key = np.zeros(points.shape[0], dtype=np.int64)
    stride = 1
    for a, n in enumerate(fine):
        key += (approximate_cell(points[:, a], AxisFold(n)) // side) * stride
        stride *= -(-n // side)
    return key, stride


def stable_order(keys: np.ndarray, bins: int):
    """(permutation, bin offsets with the trailing total)."""
    perm = np.argsort(keys, kind="stable").astype(np.int64)
    counts = np.bincount(keys, minlength=bins)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return perm, offsets


def start_in_bin(start, low, side, n):
    """start_in_bin (src/gpu_nd_bins.rs:658-670)."""
    span = np.minimum(low + side, n) - 1 - low
    delta = np.where(start < 0, start + n, start) - low
    delta = np.where(delta < 0, delta + n, delta)
    delta = np.where((delta > span) & (n - delta < delta - span), delta - n, delta)
    return start + np.clip(delta, 0, span) - delta


def prepared_slots(points: np.ndarray, fine, width: int, sides, perm, keys):
    """Prepared starts ((d + 1) int32 per slot) and offsets (d (hi, lo) pairs)
    of src/gpu_nd_bins.rs:590-709 for the stable order `perm`."""
    d = len(fine)
    points = np.asarray(points, dtype=F).reshape(-1, d)[perm]
    reach = np.all(in_reach(points), axis=1)
    rest = np.asarray(keys)[perm].copy()
    starts = np.zeros((len(perm), d + 1), dtype=np.int64)
    offsets = np.zeros((len(perm), d, 2), dtype=F)
    for a, n in enumerate(fine):
        bins_a = -(-n // sides[a])
        bin_a = rest if a == d - 1 else rest % bins_a
        rest = rest // bins_a
        start, oh, ol = support(points[:, a], AxisFold(n), width)
        start = np.where(reach, start, 0)
        starts[:, a] = start_in_bin(start, bin_a * sides[a], sides[a], n)
        offsets[:, a, 0] = np.where(reach, oh, F(1024.0))
        offsets[:, a, 1] = np.where(reach, ol, F(0.0))
    starts[:, d] = perm
    return starts.astype(np.int32), offsets
