"""Shared fixtures: the repository root on sys.path, the gpu marker, seeded inputs."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def golden():
    return np.load(ROOT / "tests" / "golden" / "direct_sums.npz")


def rel_l2(actual, expected) -> float:
    actual = np.asarray(actual)
    expected = np.asarray(expected)
    return float(np.linalg.norm(actual - expected) / np.linalg.norm(expected))


def uniform_points(rng, count, dims, dtype=np.float32):
    return rng.uniform(-np.pi, np.pi, (count, dims)).astype(dtype)


def clustered_points(rng, count, dims, centres=8, spread=0.01, dtype=np.float32):
    """Points around `centres` uniform centres with N(0, spread^2) offsets, wrapped
    into [-pi, pi) (the clustered variant of the 2D 1024^2 workload)."""
    c = rng.uniform(-np.pi, np.pi, (centres, dims))
    which = rng.integers(0, centres, count)
    p = c[which] + spread * rng.standard_normal((count, dims))
    p = (p + np.pi) % (2 * np.pi) - np.pi
    return p.astype(dtype)


def complex_normal(rng, shape, dtype=np.complex64):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
