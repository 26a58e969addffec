"""GPU parity of type-3 plans against FP64 direct sums (within 100 eps,
tests/gpu_nufft_type3.rs:13-14) and the reference's golden vectors."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import native
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402

DEV = "cuda:0"


def run_type3(sources, targets, strengths, source_bounds, target_bounds, eps, isign=1,
              precision=w.Precision.F64):
    batch = strengths.shape[0]
    config = w.NufftType3Config(tuple(map(tuple, source_bounds)), tuple(map(tuple, target_bounds)),
                                eps=eps, isign=isign, batch=batch, precision=precision)
    plan = w.NufftType3Plan(config)
    if precision == w.Precision.F32:
        rdt, cdt = torch.float32, torch.complex64
    else:
        rdt, cdt = torch.float64, torch.complex128
    src = torch.from_numpy(np.ascontiguousarray(sources)).to(DEV, rdt)
    tgt = torch.from_numpy(np.ascontiguousarray(targets)).to(DEV, rdt)
    c = torch.from_numpy(np.ascontiguousarray(strengths)).to(DEV, cdt)
    out = torch.empty((batch, targets.shape[0]), dtype=cdt, device=DEV)
    plan.encode_gpu_batch(batch, src, c, tgt, out)
    torch.cuda.synchronize()
    return out.cpu().numpy(), plan


def test_type3_matches_reference_golden(golden):
    sources, targets = golden["t3_sources"], golden["t3_targets"]
    strengths = golden["t3_strengths"]
    got, _ = run_type3(sources, targets, strengths, [[-1.0, 2.0], [0.5, 1.5]],
                       [[-20.0, 10.0], [-8.0, 8.0]], 1e-10, isign=-1)
    assert rel_l2(got, golden["t3_out"]) < 100 * 1e-10


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("eps", [1e-6, 1e-9])
def test_type3_matches_direct_sums(d, eps):
    rng = np.random.default_rng([d, int(-np.log10(eps))])
    sb = np.array([[-1.0, 1.0], [0.5, 2.5], [-3.0, -1.0]][:d])
    tb = np.array([[-40.0, 40.0], [-10.0, 30.0], [5.0, 25.0]][:d])
    sources = rng.uniform(sb[:, 0], sb[:, 1], (3000, d))
    targets = rng.uniform(tb[:, 0], tb[:, 1], (2000, d))
    strengths = rng.standard_normal((2, 3000)) + 1j * rng.standard_normal((2, 3000))
    for isign in (1, -1):
        got, plan = run_type3(sources, targets, strengths, sb, tb, eps, isign)
        ref = native.direct_type3(sources, strengths, targets, isign)
        assert rel_l2(got, ref) < 100 * eps, (isign, plan.info().outer_shape[:d])


def test_type3_metadata_matches_the_survey_configuration():
    """3D type-3 f64, sources [-1, 1]^3 -> targets [-200, 200]^3, eps 1e-9:
    the outer grid is 270^3 (2 * 2 * 200 / pi + 11 = 265.6 -> 270) and the
    inner type-2 fine grid 540^3."""
    config = w.NufftType3Config(((-1.0, 1.0),) * 3, ((-200.0, 200.0),) * 3, eps=1e-9)
    info = w.NufftType3Plan(config).info()
    assert list(info.outer_shape[:3]) == [270, 270, 270]
    assert list(info.inner_fine_shape[:3]) == [540, 540, 540]
    assert info.kernel_width == 10


def test_type3_single_source_analytic():
    """One unit source at x0: f(s) = exp(i isign s.x0) (src/type3.rs:934-963)."""
    x0 = np.array([[0.3, -0.2]])
    targets = np.random.default_rng(1).uniform(-50, 50, (500, 2))
    got, _ = run_type3(x0, targets, np.ones((1, 1), complex), [[-1, 1], [-1, 1]], [[-50, 50], [-50, 50]],
                       1e-10, isign=1)
    expected = np.exp(1j * targets @ x0[0])
    assert np.max(np.abs(got[0] - expected)) < 1e-8


def test_type3_f32_and_df64():
    rng = np.random.default_rng(3)
    sb = np.array([[-2.0, 2.0], [-1.0, 1.0]])
    tb = np.array([[-30.0, 30.0], [-30.0, 30.0]])
    sources = rng.uniform(sb[:, 0], sb[:, 1], (2000, 2))
    targets = rng.uniform(tb[:, 0], tb[:, 1], (1500, 2))
    strengths = rng.standard_normal((1, 2000)) + 1j * rng.standard_normal((1, 2000))
    ref = native.direct_type3(sources, strengths, targets, 1)
    got32, _ = run_type3(sources.astype(np.float32), targets.astype(np.float32), strengths.astype(np.complex64),
                         sb, tb, 1e-5, precision=w.Precision.F32)
    ref32 = native.direct_type3(sources.astype(np.float32).astype(np.float64), strengths,
                                targets.astype(np.float32).astype(np.float64), 1)
    assert rel_l2(got32, ref32) < 100 * 1e-5
    got64, _ = run_type3(sources, targets, strengths, sb, tb, 1e-11)
    assert rel_l2(got64, ref) < 100 * 1e-11


@pytest.mark.parametrize("d", [1, 2])
def test_type3_f32_small_outer_grids(d):
    """The regime of the reference's dense small-grid spreader
    (src/gpu_dense_spread.rs:68-78: F32, one or two axes, at most 2^16 outer
    cells): tens of thousands of sources on a few dozen cells per axis."""
    rng = np.random.default_rng(40 + d)
    sb = np.array([[-1.0, 1.0], [-0.5, 1.5]][:d])
    tb = np.array([[-30.0, 30.0], [-20.0, 25.0]][:d])
    sources = rng.uniform(sb[:, 0], sb[:, 1], (60_000, d)).astype(np.float32)
    targets = rng.uniform(tb[:, 0], tb[:, 1], (700, d)).astype(np.float32)
    strengths = (rng.standard_normal((2, 60_000)) + 1j * rng.standard_normal((2, 60_000))).astype(np.complex64)
    got, plan = run_type3(sources, targets, strengths, sb, tb, 1e-5, precision=w.Precision.F32)
    outer = list(plan.info().outer_shape[:d])
    assert int(np.prod(outer)) <= 1 << 16 and max(outer) < 100, outer
    ref = native.direct_type3(sources.astype(np.float64), strengths.astype(np.complex128),
                              targets.astype(np.float64), 1)
    assert rel_l2(got, ref) < 100 * 1e-5
    again, _ = run_type3(sources, targets, strengths, sb, tb, 1e-5, precision=w.Precision.F32)
    assert np.array_equal(got, again)
