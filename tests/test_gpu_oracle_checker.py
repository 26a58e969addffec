"""The GPU FP64 direct-sum checker (oracle/gpu_direct.py) against the CPU FP64
direct sums of oracle.cpp (themselves pinned to the reference's numpy direct
sums, python/tests/direct_sums.py) on small cases of every kind, dimension,
sign and mode order. The checker is what the full-size parity tests and the
benchmark's accuracy checks compare the CUDA path with."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import gpu_direct, native
from tests.conftest import complex_normal, rel_l2, uniform_points

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

AGREEMENT = 1e-12


@pytest.mark.parametrize("n_modes", [(37,), (16, 12), (64, 64), (6, 5, 7)])
@pytest.mark.parametrize("isign", [1, -1])
@pytest.mark.parametrize("order", [0, 1])
def test_type1_and_type2_checker_agree_with_the_cpu_sums(n_modes, isign, order):
    d = len(n_modes)
    rng = np.random.default_rng([d, isign + 2, order])
    points = uniform_points(rng, 2000, d, dtype=np.float64)
    strengths = complex_normal(rng, (3, 2000), dtype=np.complex128)
    n = int(np.prod(n_modes))
    coefficients = complex_normal(rng, (3, n), dtype=np.complex128)
    select = rng.choice(n, min(n, 300), replace=False)
    got1 = gpu_direct.direct_type1(points, strengths, n_modes, isign, order, select=select)
    ref1 = native.direct_type1(points, strengths, n_modes, isign, order, select=select)
    assert rel_l2(got1, ref1) < AGREEMENT
    pick = rng.choice(2000, 250, replace=False)
    got2 = gpu_direct.direct_type2(points, coefficients, n_modes, isign, order, select=pick)
    ref2 = native.direct_type2(points, coefficients, n_modes, isign, order, select=pick)
    assert rel_l2(got2, ref2) < AGREEMENT


@pytest.mark.parametrize("d", [1, 2, 3])
def test_type3_checker_agrees_with_the_cpu_sums(d):
    rng = np.random.default_rng(40 + d)
    sources = rng.uniform(-1, 1, (3000, d))
    targets = rng.uniform(-200, 200, (400, d))
    strengths = complex_normal(rng, (1, 3000), dtype=np.complex128)
    got = gpu_direct.direct_type3(sources, strengths, targets, -1)
    ref = native.direct_type3(sources, strengths, targets, -1)
    assert rel_l2(got, ref) < AGREEMENT


def test_checker_agrees_with_the_reference_numpy_golden(golden):
    """The reference's own numpy direct sums (tests/golden/direct_sums.npz)."""
    for index in range(int(golden["count"])):
        key = f"c{index}"
        n_modes = tuple(int(n) for n in golden[key + "_n_modes"])
        isign, order = int(golden[key + "_isign"]), int(golden[key + "_order"])
        points = golden[key + "_points"]
        got1 = gpu_direct.direct_type1(points, golden[key + "_strengths"][None], n_modes, isign, order)
        assert rel_l2(got1[0], golden[key + "_type1"]) < AGREEMENT, key
        got2 = gpu_direct.direct_type2(points, golden[key + "_coefficients"][None], n_modes, isign, order)
        assert rel_l2(got2[0], golden[key + "_type2"]) < AGREEMENT, key
    got3 = gpu_direct.direct_type3(golden["t3_sources"], golden["t3_strengths"], golden["t3_targets"], -1)
    assert rel_l2(got3, golden["t3_out"]) < AGREEMENT
