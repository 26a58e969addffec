"""Executions on prepared points can be captured in a CUDA graph (after one
warm-up execution has sized the plan's buffers) and replayed with the same
bits as eager executions: type 1 (CUDA cores and tensor cores), type 2, and
type 3."""

from __future__ import annotations

import numpy as np
import pytest

from tests.conftest import uniform_points

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import wgpunufft_b200 as w  # noqa: E402

DEV = "cuda:0"


@pytest.mark.parametrize("kind,modes,batch", [(1, (64, 48), 1), (1, (64, 48), 32), (2, (64, 48), 1),
                                               (2, (64, 48), 16), (1, (24, 20, 16), 2)])
def test_captured_execution_replays_bit_for_bit(kind, modes, batch):
    rng = np.random.default_rng(kind * 100 + batch)
    m = 20000
    points = torch.from_numpy(uniform_points(rng, m, len(modes))).to(DEV)
    n = int(np.prod(modes))
    plan = (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(w.NufftConfig(modes, 1e-6, batch=batch))
    stream = torch.cuda.Stream()
    in_len, out_len = (m, n) if kind == 1 else (n, m)
    inputs = torch.complex(torch.randn((batch, in_len), device=DEV), torch.randn((batch, in_len), device=DEV))
    out = torch.empty((batch, out_len), dtype=torch.complex64, device=DEV)
    with torch.cuda.stream(stream):
        plan.set_points_gpu(points, stream=stream)
        plan.execute_gpu_batch(batch, inputs, out, stream=stream)
        stream.synchronize()
        eager = out.clone()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            plan.execute_gpu_batch(batch, inputs, out, stream=stream)
    for _ in range(3):
        out.zero_()
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(out.view(torch.int32), eager.view(torch.int32))
    plan.synchronize()
    del graph


def test_captured_type3_replays_bit_for_bit():
    rng = np.random.default_rng(9)
    src = torch.from_numpy(rng.uniform(-1, 1, (3000, 2))).to(DEV)
    tgt = torch.from_numpy(rng.uniform(-30, 30, (2000, 2))).to(DEV)
    c = torch.complex(torch.randn((1, 3000), device=DEV, dtype=torch.float64),
                      torch.randn((1, 3000), device=DEV, dtype=torch.float64))
    plan = w.NufftType3Plan(w.NufftType3Config(((-1.0, 1.0),) * 2, ((-30.0, 30.0),) * 2, eps=1e-9))
    out = torch.empty((1, 2000), dtype=torch.complex128, device=DEV)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        plan.set_points_gpu(src, tgt, stream=stream)
        plan.execute_gpu_batch(1, c, out, stream=stream)
        stream.synchronize()
        eager = out.clone()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            plan.execute_gpu_batch(1, c, out, stream=stream)
    out.zero_()
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(out.view(torch.int64), eager.view(torch.int64))
    del graph


def test_uneven_problems_in_one_graph_match_direct_sums():
    """Independent problems of uneven sizes (2D and 3D), one plan each,
    executed from one CUDA graph: a seeded sample against direct sums."""
    from oracle import native
    from tests.conftest import rel_l2
    from wgpunufft_b200 import workloads

    problems = workloads.uneven_problems(24, seed=77)
    stream = torch.cuda.Stream()
    plans, outs = [], []
    with torch.cuda.stream(stream):
        for modes, p, c in problems:
            plan = w.NufftPlan.type1_gpu(w.NufftConfig(modes, 1e-6))
            plan.set_points_gpu(p, stream=stream)
            out = torch.empty((1, int(np.prod(modes))), dtype=torch.complex64, device=DEV)
            plan.execute_gpu_batch(1, c, out, stream=stream)
            plans.append(plan)
            outs.append(out)
        stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            for plan, (modes, p, c), out in zip(plans, problems, outs):
                plan.execute_gpu_batch(1, c, out, stream=stream)
    for out in outs:
        out.zero_()
    graph.replay()
    torch.cuda.synchronize()
    rng = np.random.default_rng(1)
    for k in rng.choice(len(problems), 6, replace=False):
        modes, p, c = problems[k]
        select = rng.choice(int(np.prod(modes)), 64, replace=False)
        ref = native.direct_type1(p.cpu().numpy().astype(np.float64), c.cpu().numpy().astype(np.complex128),
                                  modes, select=select)
        bound = 20e-6 if len(modes) == 2 else 32e-6
        assert rel_l2(outs[k].cpu().numpy()[:, select], ref) < bound, (k, modes, p.shape[0])
    del graph


@pytest.mark.parametrize("kind,modes,batch,precision", [(1, (64, 48), 1, w.Precision.F32), (1, (64, 48), 32, w.Precision.F32),
                                                        (2, (64, 48), 1, w.Precision.F32), (2, (64, 48), 16, w.Precision.F32),
                                                        (1, (24, 20, 16), 2, w.Precision.F32),
                                                        (1, (40, 36), 1, w.Precision.F64), (2, (40, 36), 3, w.Precision.F64)])
def test_captured_sort_and_execution_follow_new_points(kind, modes, batch, precision):
    """The whole one-shot transform (stable bin sort, window preparation,
    spread or interpolation, FFT, deconvolution) captured in one CUDA graph
    after a warm-up of the same point count: replays on new coordinates
    written into the same buffer give the bits of eager one-shot executions
    on those coordinates."""
    rng = np.random.default_rng(kind * 1000 + batch)
    m = 20000
    real = torch.float32 if precision == w.Precision.F32 else torch.float64
    cplx = torch.complex64 if precision == w.Precision.F32 else torch.complex128
    n = int(np.prod(modes))
    in_len, out_len = (m, n) if kind == 1 else (n, m)
    plan = (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(
        w.NufftConfig(modes, 1e-6 if precision == w.Precision.F32 else 1e-9, batch=batch, precision=precision))
    points = torch.from_numpy(uniform_points(rng, m, len(modes))).to(DEV, real)
    inputs = torch.complex(torch.randn((batch, in_len), device=DEV, dtype=real),
                           torch.randn((batch, in_len), device=DEV, dtype=real))
    out = torch.empty((batch, out_len), dtype=cplx, device=DEV)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        plan.encode_gpu_batch(batch, points, inputs, out, stream=stream)
        stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            plan.encode_gpu_batch(batch, points, inputs, out, stream=stream)
    for trial in range(2):
        fresh = np.random.default_rng(trial + 5)
        points.copy_(torch.from_numpy(uniform_points(fresh, m, len(modes))).to(DEV, real))
        inputs.copy_(torch.complex(torch.randn((batch, in_len), device=DEV, dtype=real),
                                   torch.randn((batch, in_len), device=DEV, dtype=real)))
        out.zero_()
        graph.replay()
        torch.cuda.synchronize()
        replayed = out.clone()
        with torch.cuda.stream(stream):
            plan.encode_gpu_batch(batch, points, inputs, out, stream=stream)
        plan.synchronize(stream)
        assert torch.equal(replayed.view(torch.int32), out.view(torch.int32))
    del graph


def test_persistent_batch_of_uneven_problems_matches_their_own_executions():
    """Independent 2D and 3D problems (uneven sizes, uniform and clustered)
    spread by one persistent launch over a device work counter, folded and
    transformed on forked streams: every problem's modes equal its own plan's
    execution bit for bit, eagerly and replayed from a CUDA graph, and after
    some problems get new points."""
    from wgpunufft_b200 import workloads

    problems = workloads.uneven_problems(40, seed=91)
    plans, outs, refs = [], [], []
    for modes, p, c in problems:
        plan = w.NufftPlan.type1_gpu(w.NufftConfig(modes, 1e-6))
        plan.set_points_gpu(p)
        ref = torch.empty((1, int(np.prod(modes))), dtype=torch.complex64, device=DEV)
        plan.execute_gpu_batch(1, c, ref)
        plans.append(plan)
        refs.append(ref)
        outs.append(torch.zeros_like(ref))
    torch.cuda.synchronize()
    batch = w.NufftBatch(plans)
    strengths = [c for _, _, c in problems]
    batch.execute(strengths, outs)
    torch.cuda.synchronize()
    for k, (out, ref) in enumerate(zip(outs, refs)):
        assert torch.equal(out.view(torch.int32), ref.view(torch.int32)), k
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            batch.execute(strengths, outs, stream=stream)
    for out in outs:
        out.zero_()
    graph.replay()
    torch.cuda.synchronize()
    for k, (out, ref) in enumerate(zip(outs, refs)):
        assert torch.equal(out.view(torch.int32), ref.view(torch.int32)), k
    del graph
    # New points for some problems: the batch takes the new point sets.
    for k in (0, 7, 19):
        modes, p, c = problems[k]
        fresh = workloads.points("uniform", p.shape[0], len(modes), seed=500 + k)
        plans[k].set_points_gpu(fresh)
        problems[k] = (modes, fresh, c)
        plans[k].execute_gpu_batch(1, c, refs[k])
    batch.execute(strengths, outs)
    torch.cuda.synchronize()
    for k, (out, ref) in enumerate(zip(outs, refs)):
        assert torch.equal(out.view(torch.int32), ref.view(torch.int32)), k
