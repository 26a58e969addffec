"""Seeded synthetic workloads with the shapes of the reference's benchmark
configurations, generated on the GPU, and a runner for profiling them.

    python -m wgpunufft_b200.workloads CASE [--batch B] [--executes N] [--kind 1|2|both]
                                      [--method auto|cuda|tensor]

Cases:
  small     2D 64^2 modes, 1e5 uniform points, eps 1e-6
  uniform   2D 1024^2 modes, 1e7 uniform points, eps 1e-5
  clustered 2D 1024^2 modes, 1e7 points around 8 centres (N(c, 0.01^2 I), wrapped), eps 1e-5
  radial    3D 256^3 modes, 4096 spokes x 12207 samples (radius linear in [-pi, pi),
            directions uniform on the sphere, +-1e-3 jitter), eps 1e-5
  batched   2D 512^2 modes, 2e6 uniform points, eps 1e-6, --batch vectors (default 64)
  radial128 the radial case at 128^3 modes, 4096 spokes x 1526 samples (profiling size)
  uniform3d 3D 256^3 modes, 4096 x 12207 uniform points, eps 1e-5
  uniform128 3D 128^3 modes, 4096 x 1526 uniform points, eps 1e-5 (profiling size)
  type3     3D type 3 in f64: 1e6 sources uniform in [-1, 1]^3 to 1e6 targets
            uniform in [-200, 200]^3, eps 1e-9 (--kind and --batch ignored)
  type3small2d, type3small1d
            type 3 in f32 on small outer grids: 1e6 sources uniform in
            [-1, 1]^d to 1e6 targets uniform in [-30, 30]^d, eps 1e-6
  uneven    the 256 problems of uneven_problems(), type 1, one plan each
            (--kind and --batch ignored)

uneven_problems() gives 256 independent problems of uneven sizes (2D or 3D,
modes from 64^2, 128^2, 256^2, 32^3, 64^3, M log-uniform in [1e3, 1e6],
uniform or clustered points, eps 1e-6).

Points are f32 point-major in [-pi, pi); strengths and modes complex64 with
N(0, 1) real and imaginary parts. No external dataset is involved.
"""

from __future__ import annotations

import argparse
import math

# (modes, points, eps, distribution); the type-3 entries list their outer
# grid, and "uneven" stands for its 256 problems.
CASES = {
    "small": ((64, 64), 100_000, 1e-6, "uniform"),
    "uniform": ((1024, 1024), 10_000_000, 1e-5, "uniform"),
    "clustered": ((1024, 1024), 10_000_000, 1e-5, "clustered"),
    "radial": ((256, 256, 256), 4096 * 12207, 1e-5, "radial"),
    "batched": ((512, 512), 2_000_000, 1e-6, "uniform"),
    "radial128": ((128, 128, 128), 4096 * 1526, 1e-5, "radial"),
    "uniform3d": ((256, 256, 256), 4096 * 12207, 1e-5, "uniform"),
    "uniform128": ((128, 128, 128), 4096 * 1526, 1e-5, "uniform"),
    "type3": ((270, 270, 270), 1_000_000, 1e-9, "uniform"),
    "type3small1d": ((48,), 1_000_000, 1e-6, "uniform"),
    "type3small2d": ((48, 48), 1_000_000, 1e-6, "uniform"),
    "uneven": ((64, 64), 0, 1e-6, "uniform"),
}


def points(kind: str, count: int, dims: int, seed: int = 7, device: str = "cuda"):
    """Seeded f32 points (count, dims) of the given distribution on `device`."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    two_pi = 2.0 * math.pi
    if kind == "uniform":
        p = torch.rand((count, dims), generator=g, device=device, dtype=torch.float64) * two_pi - math.pi
    elif kind == "clustered":
        centres = torch.rand((8, dims), generator=g, device=device, dtype=torch.float64) * two_pi - math.pi
        which = torch.randint(0, 8, (count,), generator=g, device=device)
        p = centres[which] + 0.01 * torch.randn((count, dims), generator=g, device=device, dtype=torch.float64)
        p = torch.remainder(p + math.pi, two_pi) - math.pi
    elif kind == "radial":
        spokes, per = 4096, count // 4096
        v = torch.randn((spokes, 3), generator=g, device=device, dtype=torch.float64)
        v = v / v.norm(dim=1, keepdim=True)
        r = torch.linspace(-math.pi, math.pi, per + 1, device=device, dtype=torch.float64)[:-1]
        p = (v[:, None, :] * r[None, :, None]).reshape(-1, 3)
        p = p + (torch.rand(p.shape, generator=g, device=device, dtype=torch.float64) * 2e-3 - 1e-3)
        p = torch.clamp(p, -math.pi, math.pi - 1e-6)
    else:
        raise ValueError(f"unknown point distribution {kind!r}")
    return p.to(torch.float32).contiguous()


def values(batch: int, count: int, seed: int = 8, device: str = "cuda"):
    """Seeded complex64 values (batch, count) with N(0, 1) parts."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return torch.complex(torch.randn((batch, count), generator=g, device=device),
                         torch.randn((batch, count), generator=g, device=device))


UNEVEN_MODES = ((64, 64), (128, 128), (256, 256), (32, 32, 32), (64, 64, 64))


def uneven_problems(count: int = 256, seed: int = 5, device: str = "cuda"):
    """Independent type-1 problems of uneven sizes: dimensions 2D or 3D with
    equal odds, modes from UNEVEN_MODES of that dimension, M log-uniform in
    [1e3, 1e6], uniform or clustered points with equal odds, eps 1e-6.
    Returns a list of (modes, points, strengths) on `device`."""
    import numpy as np

    rng = np.random.default_rng(seed)
    problems = []
    for k in range(count):
        dims = 2 if rng.random() < 0.5 else 3
        choices = [m for m in UNEVEN_MODES if len(m) == dims]
        modes = choices[int(rng.integers(len(choices)))]
        m = int(round(10 ** rng.uniform(3.0, 6.0)))
        dist = "uniform" if rng.random() < 0.5 else "clustered"
        p = points(dist, m, dims, seed=seed * 1000 + 2 * k)
        c = values(1, m, seed=seed * 1000 + 2 * k + 1)
        problems.append((modes, p, c))
    return problems


def run_type3(executes: int) -> None:
    import torch

    import wgpunufft_b200 as w

    g = torch.Generator(device="cuda")
    g.manual_seed(51)
    src = (torch.rand((1_000_000, 3), generator=g, device="cuda", dtype=torch.float64) * 2 - 1).contiguous()
    tgt = (torch.rand((1_000_000, 3), generator=g, device="cuda", dtype=torch.float64) * 400 - 200).contiguous()
    c = torch.complex(torch.randn((1, 1_000_000), generator=g, device="cuda", dtype=torch.float64),
                      torch.randn((1, 1_000_000), generator=g, device="cuda", dtype=torch.float64))
    plan = w.NufftType3Plan(w.NufftType3Config(((-1.0, 1.0),) * 3, ((-200.0, 200.0),) * 3, eps=1e-9))
    out = torch.empty((1, 1_000_000), dtype=torch.complex128, device="cuda")
    plan.set_points_gpu(src, tgt)
    for _ in range(executes):
        plan.execute_gpu_batch(1, c, out)
    torch.cuda.synchronize()


def run_type3_small(d: int, executes: int) -> None:
    import torch

    import wgpunufft_b200 as w

    g = torch.Generator(device="cuda")
    g.manual_seed(60 + d)
    src = (torch.rand((1_000_000, d), generator=g, device="cuda") * 2 - 1).contiguous()
    tgt = (torch.rand((1_000_000, d), generator=g, device="cuda") * 60 - 30).contiguous()
    c = torch.complex(torch.randn((1, 1_000_000), generator=g, device="cuda"),
                      torch.randn((1, 1_000_000), generator=g, device="cuda"))
    config = w.NufftType3Config(((-1.0, 1.0),) * d, ((-30.0, 30.0),) * d, eps=1e-6, precision=w.Precision.F32)
    plan = w.NufftType3Plan(config)
    out = torch.empty((1, 1_000_000), dtype=torch.complex64, device="cuda")
    plan.set_points_gpu(src, tgt)
    for _ in range(executes):
        plan.execute_gpu_batch(1, c, out)
    torch.cuda.synchronize()


def run(case: str, batch: int, executes: int, kinds, method: int = 0) -> None:
    import torch

    import wgpunufft_b200 as w

    if case == "type3":
        run_type3(executes)
        return
    if case.startswith("type3small"):
        run_type3_small(int(case[-2]), executes)
        return
    if case == "uneven":
        plans = []
        for modes, p, c in uneven_problems():
            plan = w.NufftPlan.type1_gpu(w.NufftConfig(modes, 1e-6))
            plan.set_points_gpu(p)
            n = 1
            for m in modes:
                n *= m
            plans.append((plan, c, torch.empty((1, n), dtype=torch.complex64, device="cuda")))
        for _ in range(executes):
            for plan, c, out in plans:
                plan.execute_gpu_batch(1, c, out)
        torch.cuda.synchronize()
        return

    modes, count, eps, dist = CASES[case]
    p = points(dist, count, len(modes))
    n = 1
    for m in modes:
        n *= m
    for kind in kinds:
        config = w.NufftConfig(modes, eps, batch=batch, spread_method=method)
        plan = (w.NufftPlan.type1_gpu if kind == 1 else w.NufftPlan.type2_gpu)(config)
        plan.set_points_gpu(p)
        inputs = values(batch, count if kind == 1 else n)
        out = torch.empty((batch, n if kind == 1 else count), dtype=torch.complex64, device="cuda")
        for _ in range(executes):
            plan.execute_gpu_batch(batch, inputs, out)
        plan.synchronize()
        del plan, inputs, out
    torch.cuda.synchronize()


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("case", choices=sorted(CASES))
    parser.add_argument("--batch", type=int, default=None)
    parser.add_argument("--executes", type=int, default=2)
    parser.add_argument("--kind", choices=["1", "2", "both"], default="both")
    parser.add_argument("--method", choices=["auto", "cuda", "tensor"], default="auto",
                        help="spreading / interpolation engine (the plan's spread_method)")
    args = parser.parse_args()
    batch = args.batch if args.batch is not None else (64 if args.case == "batched" else 1)
    kinds = (1, 2) if args.kind == "both" else (int(args.kind),)
    method = {"auto": 0, "cuda": 1, "tensor": 2}[args.method]
    run(args.case, batch, args.executes, kinds, method)
    print("ok")


if __name__ == "__main__":
    main()

