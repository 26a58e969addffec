"""Generates tests/golden/direct_sums.npz from the reference's own Python direct sums.

The reference ships FP64 direct type-1/2/3 sums in numpy
(python/tests/direct_sums.py); this script imports that file from a checkout
of the reference (the first argument, or the WGPU_NUFFT_REFERENCE environment
variable), evaluates
seeded small cases that follow the reference's tests (python/tests/test_cpu.py:
60 points, modes (11,), (6, 5), (4, 3, 5), both signs, both mode orders;
type 3 in 2D with bounds [[-1, 2], [0.5, 1.5]] -> [[-20, 10], [-8, 8]]), and
stores inputs and outputs in this package's flat layouts: modes axis-0
fastest, values transform-major. The fixtures let the oracle be pinned to the
reference without the reference present.
"""

from __future__ import annotations

import importlib.util
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def load_reference(root: Path):
    path = root / "python" / "tests" / "direct_sums.py"
    spec = importlib.util.spec_from_file_location("reference_direct_sums", path)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def to_flat(array_nd: np.ndarray) -> np.ndarray:
    """An array indexed [i0, i1, ...] as a flat axis-0-fastest vector."""
    return np.ascontiguousarray(array_nd.transpose()).reshape(-1)


def from_flat(flat: np.ndarray, n_modes) -> np.ndarray:
    return np.asarray(flat).reshape(tuple(n_modes)[::-1]).transpose()


def main(root: Path) -> None:
    ref = load_reference(root)
    cases = {}
    index = 0
    for n_modes in [(11,), (6, 5), (4, 3, 5), (16, 12)]:
        for isign in (-1, 1):
            for order in ("centered", "fft"):
                rng = np.random.default_rng([len(n_modes), isign + 1, len(order), index])
                d = len(n_modes)
                points = rng.uniform(-np.pi, np.pi, (60, d))
                strengths = rng.standard_normal(60) + 1j * rng.standard_normal(60)
                coefficients = rng.standard_normal(n_modes) + 1j * rng.standard_normal(n_modes)
                modes = ref.direct_type1(points if d > 1 else points[:, 0], strengths, n_modes, isign, order)
                values = ref.direct_type2(points if d > 1 else points[:, 0], coefficients, n_modes, isign, order)
                key = f"c{index}"
                cases[f"{key}_n_modes"] = np.array(n_modes, dtype=np.int64)
                cases[f"{key}_isign"] = np.array(isign)
                cases[f"{key}_order"] = np.array(0 if order == "centered" else 1)
                cases[f"{key}_points"] = points
                cases[f"{key}_strengths"] = strengths
                cases[f"{key}_type1"] = to_flat(modes)
                cases[f"{key}_coefficients"] = to_flat(coefficients)
                cases[f"{key}_type2"] = values
                index += 1
    cases["count"] = np.array(index)
    rng = np.random.default_rng(3)
    source_bounds = np.array([[-1.0, 2.0], [0.5, 1.5]])
    target_bounds = np.array([[-20.0, 10.0], [-8.0, 8.0]])
    sources = rng.uniform(source_bounds[:, 0], source_bounds[:, 1], (50, 2))
    targets = rng.uniform(target_bounds[:, 0], target_bounds[:, 1], (40, 2))
    strengths = rng.standard_normal((2, 50)) + 1j * rng.standard_normal((2, 50))
    cases["t3_sources"] = sources
    cases["t3_targets"] = targets
    cases["t3_strengths"] = strengths
    cases["t3_out"] = np.stack([ref.direct_type3(sources, strengths[b], targets, -1) for b in range(2)])
    np.savez_compressed(HERE / "direct_sums.npz", **cases)
    print(f"wrote {HERE / 'direct_sums.npz'} with {index} type-1/2 cases and one type-3 case")


if __name__ == "__main__":
    location = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WGPU_NUFFT_REFERENCE")
    if not location:
        sys.exit("usage: make_golden.py <reference checkout> (or set WGPU_NUFFT_REFERENCE)")
    main(Path(location))
