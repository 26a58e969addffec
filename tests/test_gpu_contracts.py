"""The reference's bit-level contracts and the small 2D configuration at its
exact size.

- Small 2D configuration (64^2 modes, 10^5 uniform points, eps 1e-6): every
  mode (type 1) and every point (type 2) against the oracle's FP64 direct
  sums over all inputs, within the reference's 2D bound of 20 eps
  (tests/gpu_nufft_2d.rs:15-16); the restated CPU plan on the same inputs
  meets the same bound.
- Batched executions equal a loop of single-vector executions bit for bit
  (tests/gpu_nufft_batch.rs:96-147) on the CUDA-core spreader and
  interpolation, in 1D, 2D and 3D. (The tensor-core paths, chosen by default
  for 2D batches of 16 or more, are held to relative l2 instead:
  tests/test_gpu_tc_spread.py, tests/test_gpu_tc_interp.py.)
- Duplicate points give bit-equal type-2 values (tests/gpu_nufft_2d.rs:149-163).
"""

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


def gpu(array):
    return torch.from_numpy(np.ascontiguousarray(array)).to(DEV)


def execute(kind, config, points, inputs, batch):
    plan = (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(config)
    m = points.shape[0]
    outputs = config.mode_count() if kind == 1 else m
    out = torch.empty((batch, outputs), dtype=torch.complex64, device=DEV)
    plan.encode_gpu_batch(batch, gpu(points), gpu(inputs.reshape(batch, -1)), out)
    plan.synchronize()
    return out.cpu().numpy()


def test_small_2d_configuration_every_output_against_direct_sums():
    """64^2 modes, 10^5 uniform points in [-pi, pi)^2, N(0, 1) complex
    strengths and modes, eps 1e-6, sigma 2: all 4,096 modes of type 1 and all
    10^5 points of type 2 against FP64 direct sums over all inputs."""
    rng = np.random.default_rng(20240611)
    modes, m, eps = (64, 64), 100_000, 1e-6
    points = uniform_points(rng, m, 2)
    strengths = complex_normal(rng, m)
    coefficients = complex_normal(rng, 64 * 64)
    config = w.NufftConfig(modes, eps)
    got1 = execute(1, config, points, strengths, 1)
    ref1 = native.direct_type1(points.astype(np.float64), strengths, modes)
    assert rel_l2(got1, ref1) < 20 * eps
    got2 = execute(2, config, points, coefficients, 1)
    ref2 = native.direct_type2(points.astype(np.float64), coefficients, modes)
    assert rel_l2(got2, ref2) < 20 * eps
    # The restated CPU plan (the timed baseline) on the same inputs.
    cpu1 = native.CpuPlan(1, modes, eps).execute(points, strengths)
    cpu2 = native.CpuPlan(2, modes, eps).execute(points, coefficients)
    assert rel_l2(cpu1, ref1) < 20 * eps
    assert rel_l2(cpu2, ref2) < 20 * eps


@pytest.mark.parametrize("n_modes", [(300,), (48, 40), (16, 16, 12)])
@pytest.mark.parametrize("batch", [3, 16])
def test_batched_equals_loop_of_single_vectors_bitwise(n_modes, batch):
    d = len(n_modes)
    rng = np.random.default_rng([d, batch])
    m = 20_000
    points = uniform_points(rng, m, d)
    strengths = complex_normal(rng, (batch, m))
    coefficients = complex_normal(rng, (batch, int(np.prod(n_modes))))
    method = w.SpreadMethod.CUDA_CORES
    many1 = execute(1, w.NufftConfig(n_modes, 1e-5, batch=batch, spread_method=method), points, strengths, batch)
    many2 = execute(2, w.NufftConfig(n_modes, 1e-5, batch=batch, spread_method=method), points, coefficients,
                    batch)
    single1 = w.NufftConfig(n_modes, 1e-5, spread_method=method)
    single2 = w.NufftConfig(n_modes, 1e-5, spread_method=method)
    for b in range(batch):
        one1 = execute(1, single1, points, strengths[b], 1)
        one2 = execute(2, single2, points, coefficients[b], 1)
        assert np.array_equal(many1[b].view(np.uint32), one1[0].view(np.uint32)), b
        assert np.array_equal(many2[b].view(np.uint32), one2[0].view(np.uint32)), b


def test_duplicate_points_give_bit_equal_type2_values():
    """tests/gpu_nufft_2d.rs:149-163: 12 x 10 modes, eps 1e-6, negative sign,
    FFT mode order; points 0-2 coincide and points 3-4 coincide."""
    points = np.array([[0.375, -1.125], [0.375, -1.125], [0.375, -1.125], [-2.25, 1.75], [-2.25, 1.75]],
                      dtype=np.float32)
    rng = np.random.default_rng(149)
    coefficients = complex_normal(rng, 120)
    config = w.NufftConfig((12, 10), 1e-6, isign=-1, mode_order=w.ModeOrder.FFT)
    got = execute(2, config, points, coefficients, 1)[0].view(np.uint32).reshape(5, 2)
    assert np.array_equal(got[1], got[0]) and np.array_equal(got[2], got[0])
    assert np.array_equal(got[4], got[3])
    # The same inside a large point set, in 1D, 2D and 3D.
    for d, n_modes in ((1, (200,)), (2, (64, 48)), (3, (24, 20, 16))):
        pts = uniform_points(rng, 50_000, d)
        pts[1::1000] = pts[0::1000][: len(pts[1::1000])]
        f = complex_normal(rng, int(np.prod(n_modes)))
        vals = execute(2, w.NufftConfig(n_modes, 1e-5), pts, f, 1)[0].view(np.uint64)
        assert np.array_equal(vals[1::1000], vals[0::1000][: len(vals[1::1000])]), d
