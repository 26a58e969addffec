"""The benchmark configurations at their full sizes: accuracy on seeded
subsets against FP64 direct sums, and size-independent properties (bitwise
repeatability over 10 runs, linearity, batch consistency)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import gpu_direct
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402
from wgpunufft_b200 import workloads  # noqa: E402

DEV = "cuda:0"


def _plan(kind, modes, eps, batch=1, method=0):
    config = w.NufftConfig(modes, eps, batch=batch, spread_method=method)
    return (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(config)


def test_2d_clustered_ten_million_points_repeatable_over_ten_runs():
    """2D 1024^2 modes, 10^7 clustered points, eps 1e-5: type-1 output bits are
    identical over 10 executions and over a fresh sort of the same points."""
    modes, count, eps, dist = workloads.CASES["clustered"]
    p = workloads.points(dist, count, 2, seed=21)
    c = workloads.values(1, count, seed=22)
    plan = _plan(1, modes, eps)
    plan.set_points_gpu(p)
    out = torch.empty((1, modes[0] * modes[1]), dtype=torch.complex64, device=DEV)
    plan.execute_gpu_batch(1, c, out)
    first = out.clone()
    for _ in range(9):
        plan.execute_gpu_batch(1, c, out)
        assert torch.equal(out.view(torch.int32), first.view(torch.int32))
    plan.set_points_gpu(p.clone())
    plan.execute_gpu_batch(1, c, out)
    assert torch.equal(out.view(torch.int32), first.view(torch.int32))
    select = np.sort(np.random.default_rng(5).choice(modes[0] * modes[1], 1024, replace=False))
    ref = gpu_direct.direct_type1(p, c, modes, select=select)
    assert rel_l2(first.cpu().numpy()[:, select], ref) < 20 * eps


def test_3d_radial_fifty_million_points():
    """3D 256^3 modes, 4096 x 12207 radial samples, eps 1e-5: type-1 on 1,024
    modes and type-2 on 10,000 points against direct sums over all inputs (3D
    bound 32 eps), and type-1 linearity at full size."""
    modes, count, eps, dist = workloads.CASES["radial"]
    p = workloads.points(dist, count, 3, seed=31)
    c = workloads.values(1, count, seed=32)
    n = modes[0] * modes[1] * modes[2]
    plan1 = _plan(1, modes, eps)
    plan1.set_points_gpu(p)
    out = torch.empty((1, n), dtype=torch.complex64, device=DEV)
    plan1.execute_gpu_batch(1, c, out)
    got = out.cpu().numpy()
    rng = np.random.default_rng(6)
    select = np.sort(rng.choice(n, 1024, replace=False))
    ref = gpu_direct.direct_type1(p, c, modes, select=select)
    assert rel_l2(got[:, select], ref) < 32 * eps
    # Linearity: T(2 c + c') = 2 T(c) + T(c').
    c2 = workloads.values(1, count, seed=33)
    out2 = torch.empty_like(out)
    plan1.execute_gpu_batch(1, c2, out2)
    mix = torch.empty_like(out)
    plan1.execute_gpu_batch(1, 2 * c + c2, mix)
    assert rel_l2(mix.cpu().numpy(), 2 * got + out2.cpu().numpy()) < 1e-5
    del plan1, out, out2, mix
    plan2 = _plan(2, modes, eps)
    plan2.set_points_gpu(p)
    f = workloads.values(1, n, seed=34)
    values = torch.empty((1, count), dtype=torch.complex64, device=DEV)
    plan2.execute_gpu_batch(1, f, values)
    pick = np.sort(rng.choice(count, 10_000, replace=False))
    ref2 = gpu_direct.direct_type2(p, f, modes, select=pick)
    assert rel_l2(values.cpu().numpy()[:, pick], ref2) < 32 * eps


def test_batched_256_vectors_tensor_cores_match_cuda_cores():
    """2D 512^2 modes, 2*10^6 points, 256 vectors, eps 1e-6: the tensor-core
    spread against direct sums (rel-l2 <= 1e-5) and against the CUDA-core
    spreader on every vector."""
    modes, count, eps, dist = workloads.CASES["batched"]
    p = workloads.points(dist, count, 2, seed=41)
    c = workloads.values(256, count, seed=42)
    n = modes[0] * modes[1]
    outs = []
    for method in (w.SpreadMethod.TENSOR_CORES, w.SpreadMethod.CUDA_CORES):
        plan = _plan(1, modes, eps, batch=256, method=method)
        plan.set_points_gpu(p)
        out = torch.empty((256, n), dtype=torch.complex64, device=DEV)
        plan.execute_gpu_batch(256, c, out)
        outs.append(out.cpu().numpy())
        del plan, out
    tensor, cuda = outs
    assert rel_l2(tensor, cuda) < 5e-6
    select = np.sort(np.random.default_rng(7).choice(n, 1024, replace=False))
    ref = gpu_direct.direct_type1(p, c[::64], modes, select=select)
    assert rel_l2(tensor[::64][:, select], ref) < 1e-5


def test_type3_3d_f64_million_sources_to_million_targets():
    """3D type-3 f64: 10^6 sources in [-1, 1]^3 to 10^6 targets in
    [-200, 200]^3, eps 1e-9 (outer grid 270^3, inner 540^3): 1000 targets
    against direct sums over all sources (type-3 bound 100 eps)."""
    g = torch.Generator(device=DEV)
    g.manual_seed(51)
    src = (torch.rand((1_000_000, 3), generator=g, device=DEV, dtype=torch.float64) * 2 - 1).contiguous()
    tgt = (torch.rand((1_000_000, 3), generator=g, device=DEV, dtype=torch.float64) * 400 - 200).contiguous()
    c = torch.complex(torch.randn((1, 1_000_000), generator=g, device=DEV, dtype=torch.float64),
                      torch.randn((1, 1_000_000), generator=g, device=DEV, dtype=torch.float64))
    config = w.NufftType3Config(((-1.0, 1.0),) * 3, ((-200.0, 200.0),) * 3, eps=1e-9)
    plan = w.NufftType3Plan(config)
    info = plan.info()
    assert list(info.outer_shape[:3]) == [270, 270, 270]
    out = torch.empty((1, 1_000_000), dtype=torch.complex128, device=DEV)
    plan.encode_gpu_batch(1, src, c, tgt, out)
    torch.cuda.synchronize()
    pick = np.sort(np.random.default_rng(8).choice(1_000_000, 1000, replace=False))
    ref = gpu_direct.direct_type3(src, c, tgt, 1, select=pick)
    assert rel_l2(out.cpu().numpy()[:, pick], ref) < 100 * 1e-9
