"""GPU parity of plans with 4 to 8 dimensions (the reference's rank-generic
path, src/gpu_nd.rs and src/gpu_nd_spread.rs for d >= 4) against the FP64
direct sums: type 1 and type 2, f32 and f64, both signs and mode orders,
batches, and bitwise repeatable type-1 outputs."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import native
from tests.conftest import complex_normal, rel_l2, uniform_points

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402

DEV = "cuda:0"


def tolerance(eps: float, precision: int) -> float:
    # The reference bounds 3D at 32 eps; one more factor of two per extra
    # axis, over the f32 floor.
    return max(64.0 * eps, 5e-5 if precision == w.Precision.F32 else 0.0)


def to_gpu(array, precision):
    real = np.float32 if precision == w.Precision.F32 else np.float64
    cplx = np.complex64 if precision == w.Precision.F32 else np.complex128
    a = np.asarray(array)
    a = a.astype(cplx if np.iscomplexobj(a) else real)
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def run(kind, n_modes, eps, precision, points, inputs, isign=1, order=0, batch=1):
    config = w.NufftConfig(n_modes, eps, isign=isign, mode_order=order, batch=batch, precision=precision)
    plan = (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(config)
    cplx = torch.complex64 if precision == w.Precision.F32 else torch.complex128
    count = config.mode_count() if kind == 1 else points.shape[0]
    out = torch.empty((batch, count), dtype=cplx, device=DEV)
    plan.set_points_gpu(to_gpu(points, precision))
    plan.execute_gpu_batch(batch, to_gpu(inputs.reshape(batch, -1), precision), out)
    plan.synchronize()
    return out.cpu().numpy(), plan


CASES = [
    ((4, 3, 5, 2), 1e-6, w.Precision.F32),
    ((4, 3, 5, 2), 1e-9, w.Precision.F64),
    ((3, 4, 2, 3, 2), 1e-3, w.Precision.F32),
    ((2, 3, 2, 2, 3, 2), 1e-4, w.Precision.F64),
    ((2,) * 8, 1e-1, w.Precision.F32),
    ((3, 2, 2, 2, 2, 2, 2), 1e-2, w.Precision.F64),
]


@pytest.mark.parametrize("n_modes,eps,precision", CASES)
def test_type1_and_type2_match_direct_sums(n_modes, eps, precision):
    rng = np.random.default_rng(len(n_modes) * 7 + int(-np.log10(eps)))
    d = len(n_modes)
    m = 400
    points = uniform_points(rng, m, d, dtype=np.float64)
    strengths = complex_normal(rng, (2, m), dtype=np.complex128)
    got, plan = run(1, n_modes, eps, precision, points, strengths, batch=2)
    ref = native.direct_type1(points, strengths, n_modes)
    assert rel_l2(got, ref) < tolerance(eps, precision)
    n = int(np.prod(n_modes))
    coefficients = complex_normal(rng, (2, n), dtype=np.complex128)
    got2, _ = run(2, n_modes, eps, precision, points, coefficients, batch=2)
    ref2 = native.direct_type2(points, coefficients, n_modes)
    assert rel_l2(got2, ref2) < tolerance(eps, precision)


@pytest.mark.parametrize("isign,order", [(-1, 0), (1, 1), (-1, 1)])
def test_signs_and_mode_orders(isign, order):
    rng = np.random.default_rng(11 + order)
    n_modes = (5, 4, 3, 4)
    points = uniform_points(rng, 300, 4, dtype=np.float64)
    strengths = complex_normal(rng, (1, 300), dtype=np.complex128)
    got, _ = run(1, n_modes, 1e-6, w.Precision.F64, points, strengths, isign=isign, order=order)
    ref = native.direct_type1(points, strengths, n_modes, isign=isign, order=order)
    assert rel_l2(got, ref) < 64e-6
    coefficients = complex_normal(rng, (1, int(np.prod(n_modes))), dtype=np.complex128)
    got2, _ = run(2, n_modes, 1e-6, w.Precision.F64, points, coefficients, isign=isign, order=order)
    ref2 = native.direct_type2(points, coefficients, n_modes, isign=isign, order=order)
    assert rel_l2(got2, ref2) < 64e-6


def test_type1_is_bitwise_repeatable_and_batch_consistent():
    """Integer accumulation: executions repeat bit for bit, and a vector
    gives the same bits alone and inside a batch (crowded points included)."""
    rng = np.random.default_rng(5)
    n_modes = (6, 5, 4, 3)
    points = np.concatenate([uniform_points(rng, 2000, 4, dtype=np.float64),
                             rng.normal(0.3, 0.01, (2000, 4))])
    strengths = complex_normal(rng, (3, 4000), dtype=np.complex128)
    config = w.NufftConfig(n_modes, 1e-5, batch=3)
    plan = w.NufftPlan.type1_gpu(config)
    plan.set_points_gpu(to_gpu(points, w.Precision.F32))
    c = to_gpu(strengths, w.Precision.F32)
    out = torch.empty((3, config.mode_count()), dtype=torch.complex64, device=DEV)
    plan.execute_gpu_batch(3, c, out)
    first = out.clone()
    for _ in range(3):
        plan.execute_gpu_batch(3, c, out)
        assert torch.equal(out.view(torch.int32), first.view(torch.int32))
    single = torch.empty((1, config.mode_count()), dtype=torch.complex64, device=DEV)
    plan.execute_gpu_batch(1, c[1:2].contiguous(), single)
    assert torch.equal(single[0].view(torch.int32), first[1].view(torch.int32))
    ref = native.direct_type1(points, strengths[:1], n_modes)
    assert rel_l2(first[:1].cpu().numpy(), ref) < 5e-5


def test_empty_point_set_and_bin_queries():
    config = w.NufftConfig((3, 3, 3, 3), 1e-3)
    plan = w.NufftPlan.type1_gpu(config)
    plan.set_points_gpu(torch.empty((0, 4), dtype=torch.float32, device=DEV))
    out = torch.full((1, 81), 7.0, dtype=torch.complex64, device=DEV)
    plan.execute_gpu_batch(1, torch.empty((1, 0), dtype=torch.complex64, device=DEV), out)
    plan.synchronize()
    assert torch.count_nonzero(out).item() == 0
    with pytest.raises(w.NufftError):
        plan.bin_order()


def test_numpy_interface_takes_five_dimensions():
    """The reference's Python plan interface on a 5D plan."""
    from wgpunufft_b200 import numpy_api as wgpu_nufft

    rng = np.random.default_rng(9)
    n_modes = (3, 2, 4, 2, 3)
    points = uniform_points(rng, 250, 5)
    strengths = complex_normal(rng, 250)
    ctx = wgpu_nufft.Context()
    plan = wgpu_nufft.Type1Plan(ctx, n_modes, eps=1e-5)
    got = plan.execute(points, strengths)
    ref = native.direct_type1(points.astype(np.float64), strengths[None, :].astype(np.complex128), n_modes)
    # The NumPy layout has the first axis slowest (shape n_modes, C order).
    d = len(n_modes)
    expected = ref.reshape(tuple(reversed(n_modes))).transpose(tuple(range(d - 1, -1, -1)))
    assert np.asarray(got).shape == n_modes
    assert rel_l2(np.asarray(got), expected) < 64e-5
