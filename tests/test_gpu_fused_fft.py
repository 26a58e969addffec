"""The fused f32 transforms of 2D and 3D plans (type 1: fold + pass along
axis 0, passes along the other axes, the last with the deconvolution; type
2: predeconvolution + pass along the last axis, ..., pass along axis 0)
against the cuFFT path of the same plans and against FP64 direct sums.

Both paths spread and interpolate the same way; they differ only in the
rounding of the FFT, so their outputs agree to a few f32 ulps of the largest
mode (relative l2 below 2e-6 at the default upsampling factor 2; below 2e-5
at 1.25 and 1.5, where the edge modes' deconvolution amplitudes amplify the
rounding of both paths), and each stays within the reference's
accuracy bars of the direct sums (20 eps in 2D, tests/gpu_nufft_2d.rs:15-16;
32 eps in 3D, tests/gpu_nufft_3d.rs:14-15).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import native
from tests.conftest import complex_normal, rel_l2, uniform_points, clustered_points

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402
from wgpunufft_b200 import _native  # noqa: E402

DEV = "cuda:0"


def set_fused(enable: bool) -> None:
    assert _native.library().b200nufft_set_fused_transforms(1 if enable else 0) == 0


@pytest.fixture(autouse=True)
def _restore_fused():
    yield
    set_fused(True)


def run(kind, modes, eps, points, values, isign, order, batch, fused, sigma=2.0):
    set_fused(fused)
    config = w.NufftConfig(modes, eps, isign=isign, mode_order=order, batch=batch, sigma=sigma)
    plan = (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(config)
    set_fused(True)
    n = config.mode_count()
    m = points.shape[0]
    out = torch.empty((batch, n if kind == 1 else m), dtype=torch.complex64, device=DEV)
    p = torch.from_numpy(np.ascontiguousarray(points)).to(DEV)
    v = torch.from_numpy(np.ascontiguousarray(values.reshape(batch, -1))).to(DEV)
    plan.set_points_gpu(p)
    plan.stage_timing(True)
    plan.execute_gpu_batch(batch, v, out)
    plan.synchronize()
    stages = plan.stage_report()
    plan.stage_timing(False)
    return out.cpu().numpy(), stages, plan.fine_grid_shape()


def power_of_two(n: int) -> bool:
    return n & (n - 1) == 0


CASES = [
    # modes, points, eps, isign, mode order, batch, distribution[, upsampling factor]
    ((203, 407), 80_000, 1e-5, 1, 1, 1, "uniform", 1.25),
    ((339, 170), 60_000, 1e-5, -1, 0, 2, "clustered", 1.5),
    ((101, 102, 203), 150_000, 1e-3, 1, 1, 1, "uniform", 1.25),
    ((64, 32, 31), 120_000, 1e-5, 1, 0, 1, "uniform"),
    ((31, 64, 64), 100_000, 1e-6, -1, 1, 2, "clustered"),
    ((128, 127, 32), 150_000, 1e-4, -1, 0, 1, "uniform"),
    ((128, 256), 60_000, 1e-5, 1, 0, 1, "uniform"),
    ((256, 128), 50_000, 1e-6, -1, 1, 2, "uniform"),
    ((127, 255), 40_000, 1e-4, 1, 1, 1, "clustered"),
    ((512, 512), 200_000, 1e-5, -1, 0, 1, "uniform"),
    ((64, 2048), 80_000, 1e-5, 1, 0, 3, "uniform"),
    ((32, 31), 5_000, 1e-6, 1, 0, 2, "uniform"),
]


@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("case", CASES,
                         ids=lambda c: "x".join(map(str, c[0])) + f"_b{c[5]}_s{c[3]}_o{c[4]}" + (f"_u{c[7]}" if len(c) > 7 else ""))
def test_fused_transforms_match_cufft_and_direct_sums(kind, case):
    modes, count, eps, isign, order, batch, dist = case[:7]
    sigma = case[7] if len(case) > 7 else 2.0
    rng = np.random.default_rng(sum(modes) + count + kind)
    d = len(modes)
    points = (uniform_points(rng, count, d) if dist == "uniform" else clustered_points(rng, count, d)).astype(np.float32)
    n = int(np.prod(modes))
    values = complex_normal(rng, batch * (count if kind == 1 else n)).astype(np.complex64)
    fused, stages, fine = run(kind, modes, eps, points, values, isign, order, batch, True, sigma)
    plain, plain_stages, _ = run(kind, modes, eps, points, values, isign, order, batch, False, sigma)
    assert all(power_of_two(f) for f in fine), fine
    if kind == 1 and np.prod(fine) > 1 << 16:
        assert "deconvolution" not in stages and "fold" in stages  # fold, row and column transforms
    if kind == 2:
        assert stages["predeconvolution"][1] == 1  # one launch: predeconvolution + column transforms
    if kind == 1:
        assert "deconvolution" in plain_stages
    # Smaller upsampling factors keep modes nearer the fine grid's edge, whose
    # deconvolution amplitudes (1 / phi_hat) grow large and amplify both
    # FFTs' rounding alike.
    agree = 2e-6 if sigma == 2.0 else 2e-5
    for b in range(batch):
        assert rel_l2(fused[b], plain[b]) < agree, (b, rel_l2(fused[b], plain[b]))
    # Against FP64 direct sums, on a subset.
    total = n if kind == 1 else count
    sel = np.arange(0, total, max(1, total // 600))
    vals = values.reshape(batch, -1).astype(np.complex128)
    if kind == 1:
        ref = native.direct_type1(points, vals, modes, isign, order, select=sel)
    else:
        ref = native.direct_type2(points, vals, modes, isign, order, select=sel)
    for b in range(batch):
        err = rel_l2(fused[b][sel], ref[b])
        assert err < max((20 if d == 2 else 32) * eps, 2e-5 if d == 2 else 3e-5), (b, err)


def test_fused_transforms_repeat_bitwise_and_batches_match_single_vectors():
    modes, count, eps = (256, 512), 100_000, 1e-5
    rng = np.random.default_rng(3)
    points = uniform_points(rng, count, 2).astype(np.float32)
    values = complex_normal(rng, 3 * count).astype(np.complex64)
    batched, _, _ = run(1, modes, eps, points, values, 1, 0, 3, True)
    again, _, _ = run(1, modes, eps, points, values, 1, 0, 3, True)
    assert np.array_equal(batched.view(np.uint8), again.view(np.uint8))
    for b in range(3):
        single, _, _ = run(1, modes, eps, points, values.reshape(3, -1)[b], 1, 0, 1, True)
        assert np.array_equal(single[0].view(np.uint8), batched[b].view(np.uint8))
    n = modes[0] * modes[1]
    coefficients = complex_normal(rng, 2 * n).astype(np.complex64)
    batched2, _, _ = run(2, modes, eps, points, coefficients, -1, 1, 2, True)
    for b in range(2):
        single, _, _ = run(2, modes, eps, points, coefficients.reshape(2, -1)[b], -1, 1, 1, True)
        assert np.array_equal(single[0].view(np.uint8), batched2[b].view(np.uint8))
