"""GPU parity of the f64 and Df64 plans.

Accuracy bars follow the reference's precision tests: f64 within 20 eps at
eps 1e-9 and 40 eps at 1e-12 (tests/gpu_nufft_precision.rs:16-20), Df64
within 24 eps (tests/gpu_nufft_df64.rs:16-20), relative l2 against FP64
direct sums. The f64 bin order (native f64 fold) is compared bit for bit with
the oracle.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import binsort, es_kernel, layout, native
from tests.conftest import clustered_points, rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402

DEV = "cuda:0"


def uniform64(rng, m, d):
    return rng.uniform(-np.pi, np.pi, (m, d))


def cnormal(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def to_df64(values: np.ndarray) -> np.ndarray:
    """(hi, lo) float pairs of every f64 scalar (complex values as re, im)."""
    flat = np.ascontiguousarray(values).view(np.float64).reshape(-1)
    hi = flat.astype(np.float32)
    lo = (flat - hi.astype(np.float64)).astype(np.float32)
    return np.stack([hi, lo], axis=-1).reshape(-1)


def from_df64(pairs: np.ndarray) -> np.ndarray:
    p = pairs.reshape(-1, 2).astype(np.float64)
    return (p[:, 0] + p[:, 1]).view(np.complex128)


def run(kind, n_modes, eps, points, values, isign=1, order=0, precision=w.Precision.F64, batch=1):
    config = w.NufftConfig(n_modes, eps, isign=isign, mode_order=order, batch=batch, precision=precision)
    plan = w.NufftPlan.type1_gpu(config) if kind == 1 else w.NufftPlan.type2_gpu(config)
    m = points.shape[0]
    count = config.mode_count() if kind == 1 else m
    if precision == w.Precision.F64:
        pts = torch.from_numpy(np.ascontiguousarray(points)).to(DEV)
        vin = torch.from_numpy(np.ascontiguousarray(values)).to(DEV)
        out = torch.empty((batch, count), dtype=torch.complex128, device=DEV)
    else:
        pts = torch.from_numpy(to_df64(points)).to(DEV)
        vin = torch.from_numpy(to_df64(values)).to(DEV)
        out = torch.empty(batch * count * 4, dtype=torch.float32, device=DEV)
    plan.set_points_gpu(pts, point_count=m)
    plan.execute_gpu_batch(batch, vin, out)
    plan.synchronize()
    got = out.cpu().numpy()
    if precision != w.Precision.F64:
        got = from_df64(got).reshape(batch, count)
    return got, plan


@pytest.mark.parametrize("n_modes", [(24,), (20, 16), (12, 10, 8)])
@pytest.mark.parametrize("eps,factor", [(1e-9, 20.0), (1e-12, 40.0)])
def test_f64_matches_direct_sums(n_modes, eps, factor):
    d = len(n_modes)
    rng = np.random.default_rng([d, int(-np.log10(eps))])
    points = uniform64(rng, 2000, d)
    strengths = cnormal(rng, 2000)
    coefficients = cnormal(rng, int(np.prod(n_modes)))
    for isign in (1, -1):
        for order in (0, 1):
            got1, _ = run(1, n_modes, eps, points, strengths, isign, order)
            ref1 = native.direct_type1(points, strengths, n_modes, isign, order)
            assert rel_l2(got1, ref1) < factor * eps
            got2, _ = run(2, n_modes, eps, points, coefficients, isign, order)
            ref2 = native.direct_type2(points, coefficients, n_modes, isign, order)
            assert rel_l2(got2, ref2) < factor * eps


@pytest.mark.parametrize("n_modes", [(32, 28), (10, 12, 8)])
@pytest.mark.parametrize("eps,bound", [(1e-9, 24e-9), (1e-11, 5e-11)])
def test_df64_storage_matches_direct_sums(n_modes, eps, bound):
    """Df64 plans within the reference's bounds (tests/gpu_nufft_df64.rs:16-20:
    24 eps; 5e-11 at eps 1e-11)."""
    d = len(n_modes)
    rng = np.random.default_rng([d, int(-np.log10(eps))])
    points = uniform64(rng, 1500, d)
    strengths = cnormal(rng, 1500)
    coefficients = cnormal(rng, int(np.prod(n_modes)))
    got1, _ = run(1, n_modes, eps, points, strengths, precision=w.Precision.DF64)
    ref1 = native.direct_type1(points, strengths, n_modes)
    assert rel_l2(got1, ref1) < bound
    got2, _ = run(2, n_modes, eps, points, coefficients, precision=w.Precision.DF64)
    ref2 = native.direct_type2(points, coefficients, n_modes)
    assert rel_l2(got2, ref2) < bound


@pytest.mark.parametrize("n_modes", [(300,), (64, 64), (16, 12, 10)])
@pytest.mark.parametrize("kind", [1, 2])
def test_f64_bin_order_is_bit_exact(n_modes, kind):
    d = len(n_modes)
    rng = np.random.default_rng([kind, d])
    eps = 1e-9
    for points in (uniform64(rng, 30_000, d), clustered_points(rng, 30_000, d).astype(np.float64)):
        config = w.NufftConfig(n_modes, eps, precision=w.Precision.F64)
        plan = w.NufftPlan.type1_gpu(config) if kind == 1 else w.NufftPlan.type2_gpu(config)
        plan.set_points_gpu(torch.from_numpy(points).to(DEV))
        perm, offsets = plan.bin_order()
        fine = list(plan.fine_grid_shape())
        width = es_kernel.es_parameters(eps, 2.0)[0]
        if kind == 1:
            lay = layout.Layout(width, fine, "F64")
            assert plan.info().chosen_geometry == lay.choose_geometry(len(points))
            sides = lay.geometries[lay.choose_geometry(len(points))].side
        else:
            sides = binsort.type2_sides64(fine)
        keys, bins = binsort.type1_keys64(points, fine, width, sides)
        ref_perm, ref_offsets = binsort.stable_order(keys, bins)
        assert np.array_equal(offsets.numpy(), ref_offsets)
        if kind == 1:
            assert np.array_equal(perm.numpy(), ref_perm)


def test_f64_bitwise_repeatable_and_batch():
    rng = np.random.default_rng(4)
    n_modes = (40, 36)
    points = uniform64(rng, 50_000, 2)
    strengths = cnormal(rng, (3, 50_000))
    first, plan = run(1, n_modes, 1e-12, points, strengths, batch=3)
    again, _ = run(1, n_modes, 1e-12, points, strengths, batch=3)
    assert np.array_equal(first.view(np.uint64), again.view(np.uint64))
    for b in range(3):
        one, _ = run(1, n_modes, 1e-12, points, strengths[b])
        assert rel_l2(first[b], one[0]) < 1e-14


def test_df64_point_count_follows_the_tensor_bytes_and_sizes_are_checked():
    """A Df64 coordinate tensor holds two floats per coordinate: the point
    count the wrapper derives from it is bytes / (dimensions x 8), the same as
    an explicit count; tensors smaller than the plan needs are rejected before
    anything reaches the device."""
    rng = np.random.default_rng(88)
    n_modes = (20, 16)
    points = uniform64(rng, 5000, 2)
    strengths = cnormal(rng, (1, 5000))
    explicit, _ = run(1, n_modes, 1e-9, points, strengths, precision=w.Precision.DF64)
    config = w.NufftConfig(n_modes, 1e-9, precision=w.Precision.DF64)
    plan = w.NufftPlan.type1_gpu(config)
    plan.set_points_gpu(torch.from_numpy(to_df64(points)).to(DEV))
    out = torch.empty(20 * 16 * 4, dtype=torch.float32, device=DEV)
    plan.execute_gpu_batch(1, torch.from_numpy(to_df64(strengths)).to(DEV), out)
    plan.synchronize()
    derived = from_df64(out.cpu().numpy()).reshape(1, -1)
    assert np.array_equal(derived.view(np.uint64), explicit.view(np.uint64))
    with pytest.raises(w.NufftError, match="InvalidArgument"):
        plan.execute_gpu_batch(1, torch.from_numpy(to_df64(strengths)).to(DEV), out[:100])
    with pytest.raises(w.NufftError, match="InvalidArgument"):
        plan.set_points_gpu(torch.from_numpy(to_df64(points)).to(DEV)[:10], point_count=5000)
