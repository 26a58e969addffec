"""Batched 2D type-2 interpolation on the tcgen05 tensor cores (3xTF32).

The tensor-core path must match FP64 direct sums within the reference's
batch bound (80 eps at eps 1e-5, tests/gpu_nufft_batch.rs:13-16; the
north-star bar of 1e-5 at eps 1e-6), agree with the CUDA-core interpolation
on every vector, repeat bit for bit, and handle batches that are not a
multiple of 64, grids whose column groups wrap, crowded and empty rows, and
points outside the fold's reach (zero values there).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import gpu_direct
from tests.conftest import clustered_points, complex_normal, rel_l2, uniform_points

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402

DEV = "cuda:0"


def interpolate(n_modes, eps, points, coefficients, batch, method):
    config = w.NufftConfig(n_modes, eps, batch=batch, spread_method=method)
    plan = w.NufftPlan.type2_gpu(config)
    plan.set_points_gpu(points)
    out = torch.empty((batch, points.shape[0]), dtype=torch.complex64, device=DEV)
    plan.execute_gpu_batch(batch, coefficients, out)
    plan.synchronize()
    return out, plan


@pytest.mark.parametrize("n_modes,eps,batch", [((64, 64), 1e-6, 16), ((48, 40), 1e-5, 64), ((96, 80), 1e-3, 80),
                                               ((256, 256), 1e-6, 130)])
def test_tensor_core_type2_matches_direct_sums_and_cuda_cores(n_modes, eps, batch):
    rng = np.random.default_rng([n_modes[0], batch])
    m = 60_000
    points = torch.from_numpy(uniform_points(rng, m, 2)).to(DEV)
    coefficients = torch.from_numpy(complex_normal(rng, (batch, int(np.prod(n_modes))))).to(DEV)
    tc, _ = interpolate(n_modes, eps, points, coefficients, batch, w.SpreadMethod.TENSOR_CORES)
    cuda, _ = interpolate(n_modes, eps, points, coefficients, batch, w.SpreadMethod.CUDA_CORES)
    pick = np.sort(rng.choice(m, 3000, replace=False))
    vectors = [0, batch // 2, batch - 1]
    ref = gpu_direct.direct_type2(points, coefficients[vectors], n_modes, select=pick)
    got = tc[vectors][:, torch.as_tensor(pick, device=DEV)].cpu().numpy()
    bound = max(80 * eps, 1e-5) if eps >= 1e-5 else 1e-5
    assert rel_l2(got, ref) < bound
    assert rel_l2(tc.cpu().numpy(), cuda.cpu().numpy()) < max(10 * eps, 5e-6)


def test_tensor_core_type2_repeats_bitwise_and_fills_every_vector():
    rng = np.random.default_rng(3)
    n_modes, batch = (128, 96), 100
    points = torch.from_numpy(clustered_points(rng, 200_000, 2, centres=3, spread=0.02)).to(DEV)
    coefficients = torch.from_numpy(complex_normal(rng, (batch, 128 * 96))).to(DEV)
    first, plan = interpolate(n_modes, 1e-5, points, coefficients, batch, w.SpreadMethod.TENSOR_CORES)
    out = torch.empty_like(first)
    for _ in range(3):
        plan.execute_gpu_batch(batch, coefficients, out)
        plan.synchronize()
        assert torch.equal(out.view(torch.int32), first.view(torch.int32))
    cuda, _ = interpolate(n_modes, 1e-5, points, coefficients, batch, w.SpreadMethod.CUDA_CORES)
    assert rel_l2(first.cpu().numpy(), cuda.cpu().numpy()) < 1e-5


def test_tensor_core_type2_active_batch_below_capacity_and_invalid_points():
    rng = np.random.default_rng(4)
    n_modes = (64, 48)
    pts = uniform_points(rng, 20_000, 2)
    pts[::997, 0] = np.nan
    pts[1::997, 1] = np.float32(1e30)
    points = torch.from_numpy(pts).to(DEV)
    coefficients = torch.from_numpy(complex_normal(rng, (40, 64 * 48))).to(DEV)
    config = w.NufftConfig(n_modes, 1e-5, batch=40)
    plan = w.NufftPlan.type2_gpu(config)  # batch >= 16: tensor cores by default
    plan.set_points_gpu(points)
    out = torch.empty((24, 20_000), dtype=torch.complex64, device=DEV)
    plan.execute_gpu_batch(24, coefficients[:24], out)
    plan.synchronize()
    got = out.cpu().numpy()
    bad = np.zeros(20_000, dtype=bool)
    bad[::997] = True
    bad[1::997] = True
    assert np.all(got[:, bad] == 0)
    good = np.flatnonzero(~bad)[::7]
    ref = gpu_direct.direct_type2(pts[good], coefficients[:24].cpu().numpy(), n_modes)
    assert rel_l2(got[:, good], ref) < 80 * 1e-5


def test_tensor_core_type2_at_the_batched_configuration():
    """2D 512^2 modes, 2*10^6 uniform points, 64 vectors, eps 1e-6: within
    1e-5 of FP64 direct sums on 10,000 points x 4 vectors."""
    rng = np.random.default_rng(5)
    n_modes, batch, m = (512, 512), 64, 2_000_000
    points = torch.from_numpy(uniform_points(rng, m, 2)).to(DEV)
    coefficients = torch.from_numpy(complex_normal(rng, (batch, 512 * 512))).to(DEV)
    tc, _ = interpolate(n_modes, 1e-6, points, coefficients, batch, w.SpreadMethod.TENSOR_CORES)
    pick = np.sort(rng.choice(m, 10_000, replace=False))
    vectors = [0, 21, 42, 63]
    ref = gpu_direct.direct_type2(points, coefficients[vectors], n_modes, select=pick)
    got = tc[vectors][:, torch.as_tensor(pick, device=DEV)].cpu().numpy()
    assert rel_l2(got, ref) < 1e-5
