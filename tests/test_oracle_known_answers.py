"""The oracle against the reference's own known answers and golden vectors (CPU only)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import es_kernel, layout, native
from tests.conftest import rel_l2


# tests/cpu_foundations.rs:482-500
@pytest.mark.parametrize("eps,width,beta", [
    (1.0e-1, 2, 4.40), (1.0e-2, 3, 6.78), (1.0e-3, 4, 9.52),
    (1.0e-4, 5, 11.50), (1.0e-5, 6, 13.80), (1.0e-6, 7, 16.10),
])
def test_es_parameter_table(eps, width, beta):
    w, b = es_kernel.es_parameters(eps, 2.0)
    assert w == width
    assert abs(b - beta) < 1e-13
    assert es_kernel.es_evaluate(w, b, 0.0) == 1.0
    assert es_kernel.es_evaluate(w, b, 0.5 * w) == 0.0
    assert es_kernel.es_evaluate(w, b, -0.5 * w) == 0.0
    assert abs(es_kernel.es_evaluate(w, b, 0.31) - es_kernel.es_evaluate(w, b, -0.31)) < 1e-15


def test_custom_sigma_formulas():
    # tests/cpu_foundations.rs:545-560
    sigma, eps = 1.25, 1.0e-6
    w, b = es_kernel.es_parameters(eps, sigma)
    assert w == math.ceil(math.log(1 / eps) / (math.pi * math.sqrt(1 - 1 / sigma)))
    assert abs(b - 0.97 * math.pi * w * (1 - 1 / (2 * sigma))) < 1e-13
    assert es_kernel.select_fine_grid_size(17, sigma, w) == 22


def test_fine_grid_sizes():
    # tests/cpu_foundations.rs:503-542
    w, _ = es_kernel.es_parameters(1.0e-6, 2.0)
    assert es_kernel.select_fine_grid_size(17, 2.0, w) == 36
    assert es_kernel.select_fine_grid_size(1, 2.0, w) == 14
    for modes in range(1, 128):
        n = es_kernel.select_fine_grid_size(modes, 2.0, w)
        assert n % 2 == 0 and n >= 2 * modes and n >= 2 * w
        assert es_kernel.fft_length_supported(n)
        first = max(2 * modes, 2 * w)
        first += first % 2
        for smaller in range(first, n, 2):
            assert not es_kernel.fft_length_supported(smaller)


def test_oversized_fine_grids_fail():
    # tests/cpu_foundations.rs:563-586
    w, _ = es_kernel.es_parameters(1.0e-6, 2.0)
    for modes, sigma in [(1000, 1.0e15), (1 << 31, 2.0)]:
        with pytest.raises(es_kernel.OracleError, match="FineGridTooLarge"):
            es_kernel.select_fine_grid_size(modes, sigma, w)


@pytest.mark.parametrize("eps", [1.0e-1, 1.0e-2, 1.0e-4, 1.0e-6, 1.0e-9, 1.0e-12])
def test_horner_table_accuracy(eps):
    # src/kernel.rs:413-446: Horner within 0.1 eps of the window.
    w, b = es_kernel.es_parameters(eps, 2.0)
    rows, table = es_kernel.horner_table(w, b, eps)
    assert table.shape == (rows, w)
    assert rows <= min(w + 3, 19)
    assert rows >= max(4, w - 4)
    d = np.linspace(-0.5 * w, 0.5 * w, 4001)
    worst = max(abs(es_kernel.horner_evaluate(w, table, x) - float(es_kernel.es_evaluate(w, b, x))) for x in d)
    assert worst <= 0.1 * eps


def test_horner_fourier_coefficients_integrate_the_polynomial():
    # src/kernel.rs:459-487
    w, b = es_kernel.es_parameters(1.0e-12, 2.0)
    _, table = es_kernel.horner_table(w, b, 1.0e-12)
    phi = es_kernel.centered_fourier_coefficients(w, b, 128, table)
    samples = 200_000
    dx = w / samples
    x = -0.5 * w + (np.arange(samples) + 0.5) * dx
    values = np.array([es_kernel.horner_evaluate(w, table, v) for v in x])
    for mode in [0, 1, 7, 31, 64]:
        freq = 2 * math.pi * mode / 128
        expected = float(np.sum(values * np.cos(freq * x)) * dx) * (-1 if mode % 2 else 1)
        assert abs(phi[mode] - expected) <= 2e-12


# src/gpu_nd_spread.rs:2158-2275
def test_layout_known_answers():
    w6 = es_kernel.es_parameters(1e-6, 2.0)[0]
    four = layout.Layout(w6, [64, 64, 64, 64], "F32")
    assert (four.run, four.workgroup_size, four.block, four.block_cells()) == (16, 64, [16, 4, 4, 4], 1024)
    one = layout.Layout(w6, [4096], "Df64")
    assert (one.run, one.workgroup_size, one.block) == (2, 64, [128])
    two = layout.Layout(w6, [512, 512], "F32")
    assert (two.run, two.workgroup_size, two.block) == (4, 32, [8, 16])
    finest = lambda shape: layout.Layout(w6, shape, "F32").geometries[0].side
    assert finest([2000, 2000]) == [1, 1]
    assert finest([200, 200, 200]) == [2, 1, 1]
    assert finest([32] * 4) == [2, 1, 1, 1]
    assert finest([400, 400, 400]) == [2, 2, 2]
    five = layout.Layout(w6, [24] * 5, "F32")
    assert five.block == [16, 4, 4, 2, 2]
    assert five.geometries[0].side == [2, 2, 2, 2, 2]
    three = layout.Layout(w6, [200, 200, 200], "F32")
    sides = [g.side for g in three.geometries]
    assert [2, 2, 2] in sides and [4, 4, 4] in sides and [16, 8, 8] in sides
    assert all(all(s <= 32 for s in g.side) for g in five.geometries)


def test_bin_geometry_follows_density():
    # src/gpu_nd_spread.rs:2187-2222
    w6 = es_kernel.es_parameters(1e-6, 2.0)[0]
    lay = layout.Layout(w6, [200, 200, 200], "F32")
    chosen = lambda m: lay.geometries[lay.choose_geometry(m)].side
    dense = chosen(10_000_000)
    assert all(s <= 2 for s in dense[1:])
    sparse = chosen(100_000)
    assert all(s >= 4 for s in sparse[1:])
    sparsest = chosen(1_000)
    assert all(a >= b for a, b in zip(sparsest, sparse))
    w3 = es_kernel.es_parameters(1e-3, 2.0)[0]
    for rank in (5, 6):
        assert layout.Layout(w3, [16] * rank, "F32").choose_geometry(1_000_000) == 0


@pytest.mark.parametrize("parts,expected", [
    (1, 1), (2, 2), (3, 2), (4, 2), (8, 4), (4096, 64), (16384, 128), (65535, 256), (65536, 256), (131072, 512),
])
def test_segment_length(parts, expected):
    assert layout.segment_length(parts) == expected


def test_survey_config_geometries():
    # Bin geometries of the benchmark configurations (2D 64^2 eps 1e-6, 2D
    # 1024^2 eps 1e-5, 3D 256^3 eps 1e-5, 2D 512^2 eps 1e-3 / 1e-6).
    cases = [((128, 128), 1e-6, 100_000, [1, 1]),
             ((2048, 2048), 1e-5, 10_000_000, [1, 1]),
             ((512, 512, 512), 1e-5, 49_999_872, [2, 2, 4]),
             ((1024, 1024), 1e-3, 2_000_000, [1, 1]),
             ((1024, 1024), 1e-6, 2_000_000, [1, 1])]
    for fine, eps, m, side in cases:
        w = es_kernel.es_parameters(eps, 2.0)[0]
        lay = layout.Layout(w, list(fine), "F32")
        assert lay.geometries[lay.choose_geometry(m)].side == side


def test_oracle_direct_sums_match_reference_golden(golden):
    for i in range(int(golden["count"])):
        k = f"c{i}"
        n_modes = tuple(golden[f"{k}_n_modes"])
        isign, order = int(golden[f"{k}_isign"]), int(golden[f"{k}_order"])
        x = golden[f"{k}_points"]
        t1 = native.direct_type1(x, golden[f"{k}_strengths"], n_modes, isign, order)[0]
        assert rel_l2(t1, golden[f"{k}_type1"]) < 1e-12
        t2 = native.direct_type2(x, golden[f"{k}_coefficients"], n_modes, isign, order)[0]
        assert rel_l2(t2, golden[f"{k}_type2"]) < 1e-12
    t3 = native.direct_type3(golden["t3_sources"], golden["t3_strengths"], golden["t3_targets"], -1)
    assert rel_l2(t3, golden["t3_out"]) < 1e-12


@pytest.mark.parametrize("precision,eps,tolerance", [("f32", 1e-5, 1e-3), ("f64", 1e-10, 1e-8)])
def test_oracle_cpu_plan_matches_reference_golden(golden, precision, eps, tolerance):
    # python/tests/test_cpu.py:12-60 tolerances.
    for i in range(int(golden["count"])):
        k = f"c{i}"
        n_modes = tuple(int(n) for n in golden[f"{k}_n_modes"])
        isign, order = int(golden[f"{k}_isign"]), int(golden[f"{k}_order"])
        x = golden[f"{k}_points"]
        t1 = native.CpuPlan(1, n_modes, eps, isign, order, precision=precision).execute(x, golden[f"{k}_strengths"])
        assert rel_l2(t1[0], golden[f"{k}_type1"]) < tolerance
        t2 = native.CpuPlan(2, n_modes, eps, isign, order, precision=precision).execute(x, golden[f"{k}_coefficients"])
        assert rel_l2(t2[0], golden[f"{k}_type2"]) < tolerance


def test_direct_conventions():
    # tests/cpu_foundations.rs:327-452
    out = native.direct_type1(np.zeros((2, 1)), [1.5 - 0.25j, -0.5 + 2j], (5,))[0]
    assert np.allclose(out, 1.0 + 1.75j, atol=1e-14)
    coefficients = np.zeros(5, complex)
    coefficients[4] = 1.0
    for isign in (1, -1):
        v = native.direct_type2([[0.37]], coefficients, (5,), isign)[0, 0]
        assert abs(v - np.exp(1j * isign * 2 * 0.37)) < 1e-14
    point = [[0.3, -0.4]]
    out = native.direct_type1(point, [1.0], (2, 3))[0]
    for value, (kx, ky) in zip(out, [(-1, -1), (0, -1), (-1, 0), (0, 0), (-1, 1), (0, 1)]):
        assert abs(value - np.exp(1j * (kx * 0.3 - ky * 0.4))) < 1e-14
