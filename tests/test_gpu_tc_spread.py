"""Batched 2D type-1 plans on the tensor-core spreader (3xTF32 tcgen05 MMAs):
accuracy against FP64 direct sums, bitwise repeatability, agreement with the
CUDA-core spreader that smaller active batches use, crowded tiles split into
parts, and uneven grids."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import native
from tests.conftest import clustered_points, rel_l2, uniform_points

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402

DEV = "cuda:0"


def _strengths(rng, batch, m):
    return (rng.standard_normal((batch, m)) + 1j * rng.standard_normal((batch, m))).astype(np.complex64)


def _run(plan, points, c, batch):
    p = torch.from_numpy(points).to(DEV)
    plan.set_points_gpu(p)
    cin = torch.from_numpy(c).to(DEV)
    out = torch.empty((batch, plan.config.mode_count()), dtype=torch.complex64, device=DEV)
    plan.execute_gpu_batch(batch, cin[:batch], out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _check(points, c, n_modes, eps, tolerance, select_count=300):
    batch = c.shape[0]
    plan = w.NufftPlan.type1_gpu(w.NufftConfig(n_modes, eps, batch=batch))
    got = _run(plan, points, c, batch)
    rng = np.random.default_rng(5)
    select = np.sort(rng.choice(int(np.prod(n_modes)), size=min(select_count, int(np.prod(n_modes))), replace=False))
    ref = native.direct_type1(points.astype(np.float64), c.astype(np.complex128), n_modes, 1, select=select)
    err = rel_l2(got[:, select], ref)
    assert err < tolerance, err
    return plan, got


@pytest.mark.parametrize("eps,tolerance", [(1e-3, 2e-3), (1e-6, 1e-5), (1e-7, 2e-6)])
def test_tensor_core_spread_matches_direct_sums(eps, tolerance):
    rng = np.random.default_rng(int(-np.log10(eps)))
    points = uniform_points(rng, 20000, 2)
    c = _strengths(rng, 80, 20000)  # one full group of 64 vectors and a partial one
    _check(points, c, (48, 40), eps, tolerance)


def test_tensor_core_spread_is_bitwise_repeatable_and_agrees_with_cuda_cores():
    rng = np.random.default_rng(11)
    points = uniform_points(rng, 30000, 2)
    c = _strengths(rng, 32, 30000)
    plan = w.NufftPlan.type1_gpu(w.NufftConfig((64, 64), 1e-6, batch=32))
    first = _run(plan, points, c, 32)
    again = _run(plan, points, c, 32)
    assert np.array_equal(first.view(np.uint32), again.view(np.uint32))
    # Active batches below 16 run on the CUDA-core spreader with the same tiles.
    small = _run(plan, points, c, 8)
    assert rel_l2(first[:8], small) < 2e-6


def test_crowded_tiles_split_into_parts():
    """Clustered points put thousands of points in a few tiles: more than 256
    chunks per tile, so tiles split into parts that the fold sums in order.
    The tolerance is the reference's 2D one, 20 eps (tests/gpu_nufft_2d.rs:15):
    tensor-memory accumulators sum in f32, so cells that gather tens of
    thousands of points lose more bits than the CUDA-core spreader's exact
    fixed-point sums, which the second check bounds."""
    rng = np.random.default_rng(12)
    points = clustered_points(rng, 60000, 2, centres=2, spread=0.005)
    c = _strengths(rng, 20, 60000)
    plan, got = _check(points, c, (96, 80), 1e-6, 20e-6)
    small = _run(plan, points, c, 8)
    assert rel_l2(got[:8], small) < 20e-6


def test_uneven_grid_and_partial_tiles():
    rng = np.random.default_rng(13)
    points = uniform_points(rng, 7000, 2)
    c = _strengths(rng, 17, 7000)
    _check(points, c, (50, 27), 1e-5, 1e-4)


def test_empty_and_single_point_sets():
    rng = np.random.default_rng(14)
    plan = w.NufftPlan.type1_gpu(w.NufftConfig((32, 32), 1e-6, batch=16))
    out = _run(plan, np.zeros((0, 2), np.float32), np.zeros((16, 0), np.complex64), 16)
    assert np.all(out == 0)
    points = uniform_points(rng, 1, 2)
    c = _strengths(rng, 16, 1)
    got = _run(plan, points, c, 16)
    ref = native.direct_type1(points.astype(np.float64), c.astype(np.complex128), (32, 32), 1)
    assert rel_l2(got, ref) < 1e-5


@pytest.mark.parametrize("eps", [1e-3, 1e-6])
def test_batched_type2_bins_match_single_vectors_bit_for_bit(eps):
    """Batched 2D f32 type-2 plans on the CUDA cores stage bin regions in
    shared memory; every vector equals its single-vector execution bit for
    bit."""
    rng = np.random.default_rng(int(-np.log10(eps)) + 40)
    points = np.concatenate([uniform_points(rng, 6000, 2), clustered_points(rng, 3000, 2, centres=3, spread=0.02)])
    batch, modes = 40, (48, 36)
    f = _strengths(rng, batch, modes[0] * modes[1])
    plan = w.NufftPlan.type2_gpu(w.NufftConfig(modes, eps, batch=batch, spread_method=w.SpreadMethod.CUDA_CORES))
    p = torch.from_numpy(points).to(DEV)
    plan.set_points_gpu(p)
    fin = torch.from_numpy(f).to(DEV)
    out = torch.empty((batch, len(points)), dtype=torch.complex64, device=DEV)
    plan.execute_gpu_batch(batch, fin, out)
    one = torch.empty((1, len(points)), dtype=torch.complex64, device=DEV)
    for b in (0, 17, 39):
        plan.execute_gpu_batch(1, fin[b:b + 1].contiguous(), one)
        assert torch.equal(one[0].view(torch.int32), out[b].view(torch.int32)), b
    torch.cuda.synchronize()
    ref = native.direct_type2(points.astype(np.float64), f[:4].astype(np.complex128), modes, 1)
    assert rel_l2(out[:4].cpu().numpy(), ref) < 20 * eps
