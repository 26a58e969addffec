"""The allocation-free bin-order entry point, b200nufft_bin_order_noalloc.

Callers that cannot allocate device memory (their framework owns the whole
device through its own pool, or they run where an allocation may block or
fail) use this entry point; its scratch lives in a fixed array in the
library. Its permutation and bin offsets must equal, bit for bit, those of
the allocating path (b200nufft_set_points + b200nufft_copy_bin_order), on two
calls in a row so that the contents the shared array keeps from the previous
call cannot leak into the next; a call must not change the device's free
memory; and a call without points only writes zero offsets. This file is
named so that pytest collects it last, and it runs alone in a fresh process
as well as after the other tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from tests.conftest import clustered_points, uniform_points

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402
from wgpunufft_b200 import _native  # noqa: E402

DEV = "cuda:0"
MAX_POINTS = 262144


def no_alloc_order(plan, points_gpu, count, check_free_memory=False):
    info = plan.info()
    d = info.dimensions
    fine = (ctypes.c_int64 * 3)(*[info.fine_shape[a] for a in range(d)], *([1] * (3 - d)))
    sides = (ctypes.c_int32 * 3)(*[info.geometry_sides[info.chosen_geometry][a] for a in range(d)],
                                 *([1] * (3 - d)))
    bins = 1
    for a in range(d):
        bins *= -(-info.fine_shape[a] // sides[a])
    perm = torch.full((max(count, 1),), -1, dtype=torch.int32, device=DEV)
    offsets = torch.full((bins + 1,), -1, dtype=torch.int32, device=DEV)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    status = _native.library().b200nufft_bin_order_noalloc(
        d, fine, info.kernel_width, sides, count, points_gpu.data_ptr() if count else None,
        perm.data_ptr(), offsets.data_ptr(), stream)
    torch.cuda.synchronize()
    if check_free_memory:
        # The call allocates nothing: the device's free memory is unchanged.
        assert torch.cuda.mem_get_info()[0] == free_before
    mask = (1 << 32) - 1
    return status, perm[:count].cpu().to(torch.int64) & mask, offsets.cpu().to(torch.int64) & mask


@pytest.mark.parametrize("n_modes", [(300,), (64, 64), (200, 150), (16, 12, 10), (40, 40, 40)])
def test_no_alloc_bin_order_matches_the_allocating_path(n_modes):
    d = len(n_modes)
    rng = np.random.default_rng([d, n_modes[0]])
    sets = [uniform_points(rng, 200_000, d), clustered_points(rng, MAX_POINTS, d), uniform_points(rng, 777, d)]
    plan = w.NufftPlan.type1_gpu(w.NufftConfig(n_modes, 1e-5))
    for points in sets:
        gpu_points = torch.from_numpy(points).to(DEV)
        plan.set_points_gpu(gpu_points)
        expected_perm, expected_offsets = plan.bin_order()
        for call in range(2):
            status, perm, offsets = no_alloc_order(plan, gpu_points, len(points), check_free_memory=call == 1)
            assert status == 0, _native.library().b200nufft_last_error()
            # A look-back that gave up would mark the trailing total 0xFFFFFFFF.
            assert int(offsets[-1]) == len(points)
            assert torch.equal(perm, expected_perm)
            assert torch.equal(offsets, expected_offsets)


def test_no_alloc_call_without_points_writes_zero_offsets():
    plan = w.NufftPlan.type1_gpu(w.NufftConfig((64, 64), 1e-5))
    plan.set_points_gpu(torch.zeros((10, 2), dtype=torch.float32, device=DEV))
    for _ in range(2):
        status, perm, offsets = no_alloc_order(plan, None, 0)
        assert status == 0, _native.library().b200nufft_last_error()
        assert perm.numel() == 0
        assert torch.count_nonzero(offsets).item() == 0


def test_no_alloc_rejects_point_counts_above_its_capacity():
    plan = w.NufftPlan.type1_gpu(w.NufftConfig((64, 64), 1e-5))
    points = torch.zeros((MAX_POINTS + 1, 2), dtype=torch.float32, device=DEV)
    plan.set_points_gpu(points[:10])
    status, _, _ = no_alloc_order(plan, points, MAX_POINTS + 1)
    assert w.STATUS_NAMES[status] == "LengthOverflow"
    assert b"262144" in _native.library().b200nufft_last_error()
