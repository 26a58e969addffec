"""ctypes wrapper of oracle/liboracle.so: FP64 direct sums and the restated CPU plan
(oracle; test infrastructure)."""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

from . import es_kernel

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "liboracle.so"

_lib = None


def build() -> Path:
    """Compiles liboracle.so with the Makefile beside this file when it is stale."""
    source = HERE / "oracle.cpp"
    if not LIBRARY.exists() or LIBRARY.stat().st_mtime < source.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIBRARY


def library():
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            build()
        _lib = ctypes.CDLL(str(LIBRARY))
    return _lib


def _i64(values):
    return np.ascontiguousarray(np.asarray(values, dtype=np.int64))


def _f64(values):
    return np.ascontiguousarray(np.asarray(values, dtype=np.float64))


def _p(array):
    return array.ctypes.data_as(ctypes.c_void_p)


def _complex_view(values, dtype):
    return np.ascontiguousarray(np.asarray(values, dtype=dtype)).view(
        np.float64 if dtype == np.complex128 else np.float32)


def direct_type1(points, strengths, n_modes, isign=1, order=0, select=None, threads=0):
    """Type-1 direct sums; `strengths` (batch, M) complex; returns (batch, count)."""
    d = len(n_modes)
    x = _f64(points).reshape(-1, d)
    c = np.atleast_2d(np.asarray(strengths, dtype=np.complex128))
    batch, m = c.shape
    sel = None if select is None else _i64(select)
    count = int(np.prod(n_modes)) if sel is None else len(sel)
    out = np.zeros((batch, count), dtype=np.complex128)
    library().oracle_direct_type1(
        ctypes.c_int(d), _p(_i64(n_modes)), ctypes.c_int(order), ctypes.c_int(1 if isign >= 0 else -1),
        ctypes.c_int64(m), _p(x), ctypes.c_int(batch), _p(np.ascontiguousarray(c)), ctypes.c_int64(count),
        None if sel is None else _p(sel), _p(out), ctypes.c_int(threads))
    return out


def direct_type2(points, coefficients, n_modes, isign=1, order=0, select=None, threads=0):
    """Type-2 direct sums; `coefficients` (batch, N) complex; returns (batch, count)."""
    d = len(n_modes)
    x = _f64(points).reshape(-1, d)
    f = np.atleast_2d(np.asarray(coefficients, dtype=np.complex128).reshape(-1, int(np.prod(n_modes))))
    batch = f.shape[0]
    sel = None if select is None else _i64(select)
    count = x.shape[0] if sel is None else len(sel)
    out = np.zeros((batch, count), dtype=np.complex128)
    library().oracle_direct_type2(
        ctypes.c_int(d), _p(_i64(n_modes)), ctypes.c_int(order), ctypes.c_int(1 if isign >= 0 else -1),
        ctypes.c_int64(x.shape[0]), _p(x), ctypes.c_int(batch), _p(np.ascontiguousarray(f)),
        ctypes.c_int64(count), None if sel is None else _p(sel), _p(out), ctypes.c_int(threads))
    return out


def direct_type3(sources, strengths, targets, isign=1, select=None, threads=0):
    """Type-3 direct sums; returns (batch, count)."""
    s = np.atleast_2d(_f64(sources))
    d = s.shape[1] if np.asarray(sources).ndim > 1 else 1
    x = _f64(sources).reshape(-1, d)
    t = _f64(targets).reshape(-1, d)
    c = np.atleast_2d(np.asarray(strengths, dtype=np.complex128))
    batch = c.shape[0]
    sel = None if select is None else _i64(select)
    count = t.shape[0] if sel is None else len(sel)
    out = np.zeros((batch, count), dtype=np.complex128)
    library().oracle_direct_type3(
        ctypes.c_int(d), ctypes.c_int(1 if isign >= 0 else -1), ctypes.c_int64(x.shape[0]), _p(x),
        ctypes.c_int(batch), _p(np.ascontiguousarray(c)), ctypes.c_int64(t.shape[0]), _p(t),
        ctypes.c_int64(count), None if sel is None else _p(sel), _p(out), ctypes.c_int(threads))
    return out


class CpuPlan:
    """The restated CpuNufftPlan for one configuration (src/cpu.rs:254-311)."""

    def __init__(self, kind: int, n_modes, eps: float, isign: int = 1, order: int = 0,
                 sigma: float = 2.0, precision: str = "f32"):
        self.kind = kind
        self.n_modes = tuple(int(n) for n in n_modes)
        self.width, self.beta = es_kernel.es_parameters(eps, sigma)
        self.fine = tuple(es_kernel.select_fine_grid_size(n, sigma, self.width) for n in self.n_modes)
        self.rows, self.table = es_kernel.horner_table(self.width, self.beta, eps)
        self.phi = [es_kernel.centered_fourier_coefficients(self.width, self.beta, n, self.table)
                    for n in self.fine]
        self.isign = 1 if isign >= 0 else -1
        self.order = order
        self.precision = precision

    def execute(self, points, values, batch: int = 1, threads: int = 0, stage_seconds=None):
        """Type 1: values (batch, M) -> modes (batch, N); type 2: (batch, N) -> (batch, M).
        An f32 plan given a list `stage_seconds` appends (prepare, execute on
        prepared points) wall times of this execution to it."""
        d = len(self.n_modes)
        real = np.float32 if self.precision == "f32" else np.float64
        ctype = np.complex64 if self.precision == "f32" else np.complex128
        pts = np.ascontiguousarray(np.asarray(points, dtype=real).reshape(-1, d))
        m = pts.shape[0]
        n = int(np.prod(self.n_modes))
        vin = np.ascontiguousarray(np.asarray(values, dtype=ctype).reshape(batch, -1))
        out = np.zeros((batch, n if self.kind == 1 else m), dtype=ctype)
        horner = np.ascontiguousarray(self.table, dtype=np.float64)
        phis = [np.ascontiguousarray(p, dtype=np.float64) for p in self.phi]
        phi_ptrs = (ctypes.c_void_p * 3)(*[_p(p) for p in phis] + [None] * (3 - d))
        args = [ctypes.c_int(self.kind), ctypes.c_int(d), _p(_i64(self.n_modes)), _p(_i64(self.fine)),
                ctypes.c_int(self.order), ctypes.c_int(self.isign), ctypes.c_int(self.width),
                ctypes.c_int(self.rows), _p(horner), phi_ptrs, ctypes.c_int(batch), ctypes.c_int64(m),
                _p(pts), _p(vin), _p(out), ctypes.c_int(threads)]
        if stage_seconds is not None and self.precision == "f32":
            seconds = np.zeros(2, dtype=np.float64)
            library().oracle_cpu_nufft_f32_timed(*args, _p(seconds))
            stage_seconds.append((float(seconds[0]), float(seconds[1])))
            return out
        fn = library().oracle_cpu_nufft_f32 if self.precision == "f32" else library().oracle_cpu_nufft_f64
        fn(*args)
        return out
