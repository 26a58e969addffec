"""GPU parity of the type-1 / type-2 CUDA path against the oracle.

Accuracy bars follow the reference's GPU tests: relative l2 error against the
FP64 direct sums within 4 eps in 1D (tests/gpu_nufft.rs:14-18), 20 eps in 2D
(tests/gpu_nufft_2d.rs:15-16) and 32 eps in 3D (tests/gpu_nufft_3d.rs:14-15),
at f32's floor of 1e-5 relative. The stable bin order, the bin offsets and
the prepared slots are compared bit for bit with the oracle's restatement of
the reference's binning.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import binsort, es_kernel, layout, native
from tests.conftest import clustered_points, complex_normal, rel_l2, uniform_points

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402

DEV = "cuda:0"


def tolerance(d: int, eps: float) -> float:
    factor = {1: 4.0, 2: 20.0, 3: 32.0}[d]
    return max(factor * eps, 2e-5 if d < 3 else 3e-5)


def to_gpu(array):
    return torch.from_numpy(np.ascontiguousarray(array)).to(DEV)


def run_type1(n_modes, eps, points, strengths, isign=1, order=0, batch=1, plan=None):
    config = w.NufftConfig(n_modes, eps, isign=isign, mode_order=order, batch=batch)
    plan = plan or w.NufftPlan.type1_gpu(config)
    n = config.mode_count()
    out = torch.empty((batch, n), dtype=torch.complex64, device=DEV)
    plan.encode_type1_gpu(to_gpu(points), to_gpu(strengths.reshape(batch, -1)), out)
    plan.synchronize()
    return out.cpu().numpy(), plan


def run_type2(n_modes, eps, points, coefficients, isign=1, order=0, batch=1, plan=None):
    config = w.NufftConfig(n_modes, eps, isign=isign, mode_order=order, batch=batch)
    plan = plan or w.NufftPlan.type2_gpu(config)
    m = points.shape[0]
    out = torch.empty((batch, m), dtype=torch.complex64, device=DEV)
    plan.encode_type2_gpu(to_gpu(points), to_gpu(coefficients.reshape(batch, -1)), out)
    plan.synchronize()
    return out.cpu().numpy(), plan


SHAPES = [(11,), (64,), (200,), (6, 5), (16, 12), (64, 64), (4, 3, 5), (16, 12, 10), (24, 20, 16)]


@pytest.mark.parametrize("n_modes", SHAPES)
@pytest.mark.parametrize("eps", [1e-3, 1e-6])
def test_type1_and_type2_match_direct_sums(n_modes, eps):
    d = len(n_modes)
    rng = np.random.default_rng([d, int(-np.log10(eps)), int(np.prod(n_modes))])
    points = uniform_points(rng, 3000, d)
    strengths = complex_normal(rng, 3000)
    coefficients = complex_normal(rng, int(np.prod(n_modes)))
    for isign in (1, -1):
        for order in (0, 1):
            got1, _ = run_type1(n_modes, eps, points, strengths, isign, order)
            ref1 = native.direct_type1(points.astype(np.float64), strengths, n_modes, isign, order)
            assert rel_l2(got1, ref1) < tolerance(d, eps), (isign, order)
            got2, _ = run_type2(n_modes, eps, points, coefficients, isign, order)
            ref2 = native.direct_type2(points.astype(np.float64), coefficients, n_modes, isign, order)
            assert rel_l2(got2, ref2) < tolerance(d, eps), (isign, order)


@pytest.mark.parametrize("eps", [1e-2, 1e-4, 1e-5])
def test_accuracy_sweep_2d(eps):
    rng = np.random.default_rng(7)
    n_modes = (32, 24)
    points = uniform_points(rng, 4000, 2)
    strengths = complex_normal(rng, 4000)
    got, _ = run_type1(n_modes, eps, points, strengths)
    ref = native.direct_type1(points.astype(np.float64), strengths, n_modes)
    assert rel_l2(got, ref) < tolerance(2, eps)


def oracle_order(points, fine, eps, kind):
    width = es_kernel.es_parameters(eps, 2.0)[0]
    if kind == 1:
        lay = layout.Layout(width, list(fine), "F32")
        side = lay.geometries[lay.choose_geometry(points.shape[0])].side
        keys, bins = binsort.type1_keys(points, fine, width, side)
    else:
        side = None
        keys, bins = binsort.type2_keys(points, fine)
    perm, offsets = binsort.stable_order(keys, bins)
    return perm, offsets, keys, side, width


def point_sets(d, rng):
    m = 20_000
    special = uniform_points(rng, m, d)
    special[::97, 0] = np.float32(np.pi)
    special[1::97, -1] = np.float32(-np.pi)
    special[2::97, 0] = np.float32(3 * np.pi)
    special[3::97, 0] = np.float32(-3 * np.pi)
    special[4::131] = special[5::131][: len(special[4::131])]  # duplicates
    special[6::211, 0] = np.nan
    special[7::211, -1] = np.inf
    special[8::211, 0] = np.float32(1e30)
    special[9::211, 0] = np.float32(5 * np.pi)
    special[10::211, 0] = np.float32(-40.0)
    return {
        "uniform": uniform_points(rng, m, d),
        "clustered": clustered_points(rng, m, d),
        "edges_and_invalid": special,
        "single_point": clustered_points(rng, 5000, d, centres=1, spread=0.0),
    }


@pytest.mark.parametrize("n_modes", [(64,), (1000,), (64, 64), (200, 150), (16, 12, 10), (40, 40, 40)])
@pytest.mark.parametrize("kind", [1, 2])
def test_bin_order_is_bit_exact(n_modes, kind):
    d = len(n_modes)
    rng = np.random.default_rng([kind, d, n_modes[0]])
    eps = 1e-5
    for name, points in point_sets(d, rng).items():
        config = w.NufftConfig(n_modes, eps)
        plan = w.NufftPlan.type1_gpu(config) if kind == 1 else w.NufftPlan.type2_gpu(config)
        gpu_points = to_gpu(points)
        plan.set_points_gpu(gpu_points)
        perm, offsets = plan.bin_order()
        fine = plan.fine_grid_shape()
        ref_perm, ref_offsets, keys, side, width = oracle_order(points, fine, eps, kind)
        assert np.array_equal(offsets.numpy(), ref_offsets), name
        assert np.array_equal(perm.numpy(), ref_perm), name
        if kind == 1:
            assert plan.info().chosen_geometry == layout.Layout(width, list(fine), "F32").choose_geometry(len(points))
            starts, offs = plan.prepared_slots()
            ref_starts, ref_offs = binsort.prepared_slots(points, fine, width, side, ref_perm, keys)
            assert np.array_equal(starts.numpy().reshape(-1, d + 1), ref_starts), name
            assert np.array_equal(offs.numpy().view(np.uint32).reshape(-1),
                                  ref_offs.reshape(-1).view(np.uint32)), name


def test_large_sort_matches_oracle():
    """A multi-tile sort (several look-back tiles and all three radix passes)."""
    rng = np.random.default_rng(11)
    for points, n_modes in [(uniform_points(rng, 3_000_000, 2), (1024, 1024)),
                            (clustered_points(rng, 2_000_000, 2), (1024, 1024)),
                            (uniform_points(rng, 1_500_000, 3), (128, 128, 128))]:
        plan = w.NufftPlan.type1_gpu(w.NufftConfig(n_modes, 1e-5))
        plan.set_points_gpu(to_gpu(points))
        perm, offsets = plan.bin_order()
        ref_perm, ref_offsets, *_ = oracle_order(points, plan.fine_grid_shape(), 1e-5, 1)
        assert np.array_equal(offsets.numpy(), ref_offsets)
        assert np.array_equal(perm.numpy(), ref_perm)


@pytest.mark.parametrize("n_modes", [(256,), (128, 128), (32, 32, 32)])
def test_bitwise_repeatable(n_modes):
    d = len(n_modes)
    rng = np.random.default_rng(5)
    points = clustered_points(rng, 200_000, d)
    strengths = complex_normal(rng, 200_000)
    coefficients = complex_normal(rng, int(np.prod(n_modes)))
    first1, plan1 = run_type1(n_modes, 1e-5, points, strengths)
    first2, plan2 = run_type2(n_modes, 1e-5, points, coefficients)
    for _ in range(10):
        again1, _ = run_type1(n_modes, 1e-5, points, strengths, plan=plan1)
        again2, _ = run_type2(n_modes, 1e-5, points, coefficients, plan=plan2)
        assert np.array_equal(first1.view(np.uint32), again1.view(np.uint32))
        assert np.array_equal(first2.view(np.uint32), again2.view(np.uint32))


@pytest.mark.parametrize("n_modes", [(128,), (48, 40), (16, 16, 12)])
def test_batch_matches_single_vectors(n_modes):
    d = len(n_modes)
    rng = np.random.default_rng(9)
    m, batch = 5000, 3
    points = uniform_points(rng, m, d)
    strengths = complex_normal(rng, (batch, m))
    coefficients = complex_normal(rng, (batch, int(np.prod(n_modes))))
    many1, _ = run_type1(n_modes, 1e-5, points, strengths, batch=batch)
    many2, _ = run_type2(n_modes, 1e-5, points, coefficients, batch=batch)
    for b in range(batch):
        one1, _ = run_type1(n_modes, 1e-5, points, strengths[b])
        one2, _ = run_type2(n_modes, 1e-5, points, coefficients[b])
        assert rel_l2(many1[b], one1[0]) < 1e-6
        assert rel_l2(many2[b], one2[0]) < 1e-6
        ref = native.direct_type1(points.astype(np.float64), strengths[b], n_modes)[0]
        assert rel_l2(many1[b], ref) < tolerance(d, 1e-5)


def test_active_batch_below_capacity_and_set_points_reuse():
    rng = np.random.default_rng(12)
    n_modes = (40, 36)
    m = 6000
    points = uniform_points(rng, m, 2)
    strengths = complex_normal(rng, (4, m))
    config = w.NufftConfig(n_modes, 1e-5, batch=4)
    plan = w.NufftPlan.type1_gpu(config)
    plan.set_points_gpu(to_gpu(points))
    out = torch.empty((2, config.mode_count()), dtype=torch.complex64, device=DEV)
    plan.execute_type1_gpu_batch(2, to_gpu(strengths[:2]), out)
    plan.synchronize()
    executed = out.cpu().numpy()
    encoded, _ = run_type1(n_modes, 1e-5, points, strengths[:2], batch=2)
    assert np.array_equal(executed.view(np.uint32), encoded.view(np.uint32))
    with pytest.raises(w.NufftError, match="InvalidBatch"):
        plan.execute_type1_gpu_batch(5, to_gpu(strengths), out)


def test_zero_points():
    n_modes = (16, 12)
    plan = w.NufftPlan.type1_gpu(w.NufftConfig(n_modes, 1e-6))
    out = torch.full((1, 192), 7.0 + 1j, dtype=torch.complex64, device=DEV)
    empty = torch.empty((0, 2), dtype=torch.float32, device=DEV)
    plan.encode_type1_gpu(empty, torch.empty((1, 0), dtype=torch.complex64, device=DEV), out)
    plan.synchronize()
    assert torch.count_nonzero(out).item() == 0
    plan2 = w.NufftPlan.type2_gpu(w.NufftConfig(n_modes, 1e-6))
    out2 = torch.empty((1, 0), dtype=torch.complex64, device=DEV)
    plan2.encode_type2_gpu(empty, torch.ones((1, 192), dtype=torch.complex64, device=DEV), out2)
    plan2.synchronize()


def test_execute_before_points_and_wrong_kind_fail():
    plan = w.NufftPlan.type1_gpu(w.NufftConfig((8,), 1e-6))
    out = torch.empty((1, 8), dtype=torch.complex64, device=DEV)
    with pytest.raises(w.NufftError, match="GpuExecutionUnavailable"):
        plan.execute_type1_gpu(out, out)
    with pytest.raises(w.NufftError, match="GpuExecutionUnavailable"):
        plan.execute_type2_gpu(out, out)


def with_invalid_points(valid, every, rng=None):
    """`valid` with a point outside the fold's reach inserted after every
    `every` points (non-finite, far, and just-outside coordinates on one axis,
    cycling; tests/gpu_invalid_points.rs:20-34); returns the mixed set and each
    mixed point's index among the valid ones (-1 for the inserted ones)."""
    d = valid.shape[1]
    invalid_values = [np.nan, np.inf, -np.inf, 1e30, -1e30, -40.0, 5 * np.pi, 1e20]
    mixed, index = [], []
    k = 0
    for i, p in enumerate(valid):
        mixed.append(p)
        index.append(i)
        if (i + 1) % every == 0:
            q = p.copy()
            q[k % d] = invalid_values[k % len(invalid_values)]
            mixed.append(q)
            index.append(-1)
            k += 1
    return np.array(mixed, dtype=valid.dtype), np.array(index)


@pytest.mark.parametrize("n_modes", [(64,), (24, 20), (16, 16, 12)])
def test_invalid_points_leave_other_points_intact(n_modes):
    """tests/gpu_invalid_points.rs: non-finite and far coordinates get zero
    weight; type-2 values at the other points are unchanged bit for bit and
    zero at the invalid ones; type-1 modes equal, bit for bit, those of the
    valid points alone, whatever the invalid points' strengths."""
    d = len(n_modes)
    rng = np.random.default_rng(21)
    valid = uniform_points(rng, 300, d)
    mixed, index = with_invalid_points(valid, 25)
    coefficients = complex_normal(rng, int(np.prod(n_modes)))
    only, _ = run_type2(n_modes, 1e-6, valid, coefficients)
    both, _ = run_type2(n_modes, 1e-6, mixed, coefficients)
    assert np.array_equal(both[0, index >= 0].view(np.uint32), only[0].view(np.uint32))
    assert np.all(both[0, index < 0] == 0)
    strengths = complex_normal(rng, len(mixed))
    strengths[index < 0] *= 1e3  # larger than every valid strength: must not set the scale
    with_invalid, _ = run_type1(n_modes, 1e-6, mixed, strengths)
    without, _ = run_type1(n_modes, 1e-6, valid, strengths[index >= 0])
    assert np.array_equal(with_invalid.view(np.uint32), without.view(np.uint32))


@pytest.mark.parametrize("n_modes,count,precision,method", [
    ((48, 40), 400_000, "f32", 1), ((16, 16, 12), 300_000, "f32", 1), ((40, 36), 200_000, "f64", 1),
    ((64, 48), 200_000, "f32", 2)])
def test_invalid_points_leave_type1_bitwise_intact_at_scale(n_modes, count, precision, method):
    """Crowded small grids above 150,000 points, where the parts are sized by
    the point count: points outside the reach change no part, no run and no
    scale, so the modes equal those of the valid points bit for bit (CUDA-core
    spreader in 2D, 3D and f64; tensor-core spreader for 16 vectors)."""
    d = len(n_modes)
    rng = np.random.default_rng(count + d)
    dtype = np.float32 if precision == "f32" else np.float64
    valid = clustered_points(rng, count, d, centres=3, spread=0.3, dtype=dtype)
    mixed, index = with_invalid_points(valid, 97)
    batch = 16 if method == 2 else 1
    cdtype = np.complex64 if precision == "f32" else np.complex128
    strengths = complex_normal(rng, (batch, len(mixed)), dtype=cdtype)
    outs = []
    for pts, st in ((mixed, strengths), (valid, np.ascontiguousarray(strengths[:, index >= 0]))):
        config = w.NufftConfig(n_modes, 1e-6 if precision == "f32" else 1e-9, batch=batch, spread_method=method,
                               precision=w.Precision.F32 if precision == "f32" else w.Precision.F64)
        plan = w.NufftPlan.type1_gpu(config)
        out = torch.empty((batch, config.mode_count()), dtype=torch.complex64 if precision == "f32" else torch.complex128,
                          device=DEV)
        plan.encode_gpu_batch(batch, to_gpu(pts), to_gpu(st), out)
        plan.synchronize()
        outs.append(out.cpu().numpy())
    view = np.uint32 if precision == "f32" else np.uint64
    assert np.array_equal(outs[0].view(view), outs[1].view(view))


def test_clustered_and_heavy_tiles_match_direct():
    """Dense clusters split tiles into many parts; the sums stay accurate."""
    rng = np.random.default_rng(31)
    n_modes = (64, 64)
    points = clustered_points(rng, 400_000, 2, centres=2, spread=0.003)
    strengths = complex_normal(rng, 400_000)
    got, _ = run_type1(n_modes, 1e-5, points, strengths)
    select = rng.choice(64 * 64, 300, replace=False)
    ref = native.direct_type1(points.astype(np.float64), strengths, n_modes, select=select)
    assert rel_l2(got[0, select], ref[0]) < tolerance(2, 1e-5)


@pytest.mark.parametrize("eps", [1e-4, 1e-5, 1e-6, 1e-7])
def test_crowded_3d_tiles_match_direct_and_repeat(eps):
    """3D tiles holding far more points than start cells (tight clusters over
    uniform background; windows 5 to 8 wide): accurate against direct sums
    and bitwise repeatable, including after a fresh sort of the points."""
    rng = np.random.default_rng(41)
    n_modes = (24, 20, 16)
    points = np.concatenate([clustered_points(rng, 150_000, 3, centres=2, spread=0.05),
                             uniform_points(rng, 50_000, 3)])
    strengths = complex_normal(rng, points.shape[0])
    got, plan = run_type1(n_modes, eps, points, strengths)
    assert 5 <= plan.kernel_width() <= 8
    again, _ = run_type1(n_modes, eps, points, strengths, plan=plan)
    assert np.array_equal(got.view(np.int32), again.view(np.int32))
    n = n_modes[0] * n_modes[1] * n_modes[2]
    select = rng.choice(n, 200, replace=False)
    ref = native.direct_type1(points.astype(np.float64), strengths, n_modes, select=select)
    assert rel_l2(got[0, select], ref[0]) < tolerance(3, eps)


def test_2d_1024_ten_million_points_against_direct_subsets():
    """The 2D 1024^2, 10^7-point workload, uniform and clustered: 1,024 seeded
    modes (type 1) and 10,000 seeded points (type 2) against FP64 direct sums
    over all inputs (the oracle's GPU checker)."""
    from oracle import gpu_direct

    rng = np.random.default_rng(2024)
    n_modes = (1024, 1024)
    m = 10_000_000
    for points in (uniform_points(rng, m, 2), clustered_points(rng, m, 2)):
        strengths = complex_normal(rng, m)
        got, plan = run_type1(n_modes, 1e-5, points, strengths)
        select = np.sort(rng.choice(1024 * 1024, 1024, replace=False))
        ref = gpu_direct.direct_type1(points, strengths[None], n_modes, select=select)
        assert rel_l2(got[0, select], ref[0]) < tolerance(2, 1e-5)
        coefficients = complex_normal(rng, 1024 * 1024)
        got2, _ = run_type2(n_modes, 1e-5, points, coefficients)
        pick = np.sort(rng.choice(m, 10_000, replace=False))
        ref2 = gpu_direct.direct_type2(points, coefficients[None], n_modes, select=pick)
        assert rel_l2(got2[0, pick], ref2[0]) < tolerance(2, 1e-5)


def test_f64_type2_staged_regions_match_the_gather_bitwise():
    """2D f64 type 2 at eps 1e-12 (w = 13): one vector runs on staged bin
    regions, a batch on the thread-per-point gather; both give the same bits,
    within the f64 bound of direct sums."""
    rng = np.random.default_rng(77)
    n_modes = (40, 36)
    points = uniform_points(rng, 3000, 2, dtype=np.float64)
    coefficients = complex_normal(rng, (2, 40 * 36), dtype=np.complex128)
    outs = []
    for batch in (1, 2):
        config = w.NufftConfig(n_modes, 1e-12, batch=batch, precision=w.Precision.F64)
        plan = w.NufftPlan.type2_gpu(config)
        plan.set_points_gpu(torch.from_numpy(points).to(DEV))
        out = torch.empty((batch, 3000), dtype=torch.complex128, device=DEV)
        plan.execute_gpu_batch(batch, torch.from_numpy(coefficients[:batch].copy()).to(DEV), out)
        plan.synchronize()
        outs.append(out.cpu().numpy())
    assert np.array_equal(outs[0][0].view(np.int64), outs[1][0].view(np.int64))
    ref = native.direct_type2(points, coefficients[:1], n_modes)
    assert rel_l2(outs[0], ref) < 20 * 1e-12 + 1e-13


def test_type2_crowded_bins_are_split_over_many_parts():
    """Type 2 on tight clusters (bins of 8 x 8 cells holding thousands of
    points, served in parts of 512 slots): one vector on the staged-region
    kernel, a batch of 40 on the batched bin kernel, and f64 on its staged
    regions give the bits of the per-point sums (the batch's first vector, the
    f64 gather) and stay within the direct-sum bound."""
    rng = np.random.default_rng(83)
    n_modes = (96, 80)
    m = 300_000
    points = np.concatenate([clustered_points(rng, m - 20_000, 2, centres=3, spread=0.004),
                             uniform_points(rng, 20_000, 2)])
    coefficients = complex_normal(rng, (40, 96 * 80))
    outs32 = []
    for batch in (1, 40):
        config = w.NufftConfig(n_modes, 1e-6, batch=batch, spread_method=w.SpreadMethod.CUDA_CORES)
        plan = w.NufftPlan.type2_gpu(config)
        assert plan.kernel_width() == 7
        plan.set_points_gpu(to_gpu(points))
        out = torch.empty((batch, m), dtype=torch.complex64, device=DEV)
        plan.execute_gpu_batch(batch, to_gpu(coefficients[:batch]), out)
        plan.synchronize()
        outs32.append(out.cpu().numpy())
    one, many = outs32
    assert np.array_equal(one[0].view(np.uint32), many[0].view(np.uint32))
    pick = np.sort(rng.choice(m, 3000, replace=False))
    for b in (0, 39):
        ref = native.direct_type2(points[pick].astype(np.float64), coefficients[b:b + 1], n_modes)
        assert rel_l2(many[b, pick], ref[0]) < tolerance(2, 1e-6)
    points64 = points.astype(np.float64)
    coefficients64 = coefficients[:2].astype(np.complex128)
    outs = []
    for batch in (1, 2):
        config = w.NufftConfig(n_modes, 1e-12, batch=batch, precision=w.Precision.F64)
        plan64 = w.NufftPlan.type2_gpu(config)
        plan64.set_points_gpu(to_gpu(points64))
        out = torch.empty((batch, m), dtype=torch.complex128, device=DEV)
        plan64.execute_gpu_batch(batch, to_gpu(coefficients64[:batch]), out)
        plan64.synchronize()
        outs.append(out.cpu().numpy())
    assert np.array_equal(outs[0][0].view(np.int64), outs[1][0].view(np.int64))
    ref64 = native.direct_type2(points64[pick], coefficients64[:1], n_modes)
    assert rel_l2(outs[0][0, pick], ref64[0]) < 20 * 1e-12 + 1e-13


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_3d_type2_bin_order_on_request_leaves_executions_alone(precision):
    """3D type-2 plans interpolate in their own point order and sort the
    reference's bins only when bin_order asks: the order is the oracle's for
    each new point set, and asking for it changes no output bit."""
    n_modes = (24, 20, 16)
    eps = 1e-5 if precision == "f32" else 1e-9
    prec = w.Precision.F32 if precision == "f32" else w.Precision.F64
    ctype = torch.complex64 if precision == "f32" else torch.complex128
    rng = np.random.default_rng(77)

    def bits(values):
        return torch.view_as_real(values).view(torch.int64 if precision == "f64" else torch.int32)

    config = w.NufftConfig(n_modes, eps, precision=prec)
    plan = w.NufftPlan.type2_gpu(config)
    coefficients = torch.from_numpy(complex_normal(rng, config.mode_count())).to(ctype).reshape(1, -1).to(DEV)
    for points in (uniform_points(rng, 30_000, 3), clustered_points(rng, 25_000, 3)):
        gpu_points = to_gpu(points if precision == "f32" else points.astype(np.float64))
        plan.set_points_gpu(gpu_points)
        out = torch.empty((1, points.shape[0]), dtype=ctype, device=DEV)
        plan.execute_gpu_batch(1, coefficients, out)
        before = out.clone()
        perm, offsets = plan.bin_order()
        if precision == "f32":
            ref_perm, ref_offsets, *_ = oracle_order(points, plan.fine_grid_shape(), eps, 2)
            assert np.array_equal(perm.numpy(), ref_perm)
        else:
            # As test_f64_bin_order_is_bit_exact: the f64 offsets against the
            # oracle, the permutation as an order of those keys.
            fine = list(plan.fine_grid_shape())
            width = es_kernel.es_parameters(eps, 2.0)[0]
            keys, bins = binsort.type1_keys64(points.astype(np.float64), fine, width, binsort.type2_sides64(fine))
            _, ref_offsets = binsort.stable_order(keys, bins)
            assert np.array_equal(np.sort(perm.numpy()), np.arange(points.shape[0]))
            assert np.all(np.diff(keys[perm.numpy()].astype(np.int64)) >= 0)
        assert np.array_equal(offsets.numpy(), ref_offsets)
        again_perm, _ = plan.bin_order()
        assert torch.equal(again_perm, perm)
        plan.execute_gpu_batch(1, coefficients, out)
        plan.synchronize()
        assert torch.equal(bits(out), bits(before))
        fresh = w.NufftPlan.type2_gpu(config)
        fresh.set_points_gpu(gpu_points)
        other = torch.empty_like(out)
        fresh.execute_gpu_batch(1, coefficients, other)
        fresh.synchronize()
        assert torch.equal(bits(other), bits(out))
