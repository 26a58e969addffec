"""FP64 direct NUFFT sums on the GPU (oracle; test infrastructure only).

ctypes wrapper of oracle/libgpu_direct.so (gpu_direct.cu). The sums are the
reference's FP64 direct oracle (src/direct.rs:9-118 for types 1 and 2,
src/type3.rs:609-673 for type 3), evaluated term by term in FP64 on the
GPU so that the full-size workloads can be checked on subsets of 10^3 to
10^4 outputs against all of their inputs. tests/test_gpu_oracle_checker.py
validates them against the CPU sums of oracle.cpp. Only tests/ and
bench.py's accuracy checks use this module; the library never does.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "libgpu_direct.so"
_lib = None
TARGET_BLOCK = 256
WAVE_BLOCKS = 148 * 8


def library():
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(f"{LIBRARY} is missing: run make -C oracle")
        _lib = ctypes.CDLL(str(LIBRARY))
        _lib.oracle_gpu_direct.restype = ctypes.c_int
        _lib.oracle_gpu_direct.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_void_p]
    return _lib


def _torch():
    import torch

    return torch


def _as_f64(x, device):
    torch = _torch()
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.ascontiguousarray(x))
    return x.to(device=device, dtype=torch.float64).contiguous()


def _as_c128(v, device):
    torch = _torch()
    if isinstance(v, np.ndarray):
        v = torch.from_numpy(np.ascontiguousarray(v))
    return v.to(device=device, dtype=torch.complex128).contiguous()


def _sums(dimensions, isign, targets, terms, values, modes=None, order=0, device="cuda:0"):
    """out[b, t] = sum_j values[b, j] exp(i isign <targets[t], terms[j]>) in FP64;
    `terms` None takes the mode grid `modes` (storage order `order`)."""
    torch = _torch()
    targets = _as_f64(targets, device).reshape(-1, dimensions)
    values = _as_c128(values, device)
    values = values.reshape(-1, values.shape[-1])
    batch, term_count = values.shape
    target_count = targets.shape[0]
    if terms is not None:
        terms = _as_f64(terms, device).reshape(-1, dimensions)
        assert terms.shape[0] == term_count
    modes_arr = (ctypes.c_int64 * 3)(*([int(n) for n in modes] if modes is not None else []), *([1] * (3 - (len(modes) if modes is not None else 0))))
    blocks = -(-target_count // TARGET_BLOCK)
    splits = int(max(1, min(1024, WAVE_BLOCKS // blocks, -(-term_count // 4096))))
    out = torch.zeros((batch, target_count), dtype=torch.complex128, device=device)
    stream = torch.cuda.current_stream(device).cuda_stream
    for b0 in range(0, batch, 4):
        group = min(4, batch - b0)
        launch = 4 if group > 2 else group
        vals = values[b0:b0 + group]
        if launch != group:
            vals = torch.cat([vals, torch.zeros((launch - group, term_count), dtype=vals.dtype, device=device)])
        vals = vals.contiguous()
        partial = torch.empty((splits, launch, target_count), dtype=torch.complex128, device=device)
        rc = library().oracle_gpu_direct(
            dimensions, launch, 1 if isign >= 0 else -1, target_count, targets.data_ptr(), term_count,
            None if terms is None else terms.data_ptr(), modes_arr, order, vals.data_ptr(), splits,
            partial.data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"oracle_gpu_direct failed with code {rc}")
        # Ranges added in split order: a fixed order.
        total = partial[0].clone()
        for s in range(1, splits):
            total += partial[s]
        out[b0:b0 + group] = total[:group]
    torch.cuda.synchronize(device)
    return out.cpu().numpy()


def mode_vectors(n_modes, order=0, select=None):
    """Integer mode vectors (as float64) of the flat storage indices `select`
    (all modes when None), axis 0 fastest (src/direct.rs:120-131)."""
    n_modes = [int(n) for n in n_modes]
    total = int(np.prod(n_modes))
    flat = np.arange(total, dtype=np.int64) if select is None else np.asarray(select, dtype=np.int64)
    out = np.empty((flat.shape[0], len(n_modes)), dtype=np.float64)
    rest = flat.copy()
    for a, n in enumerate(n_modes):
        index = rest % n
        rest //= n
        if order == 0:
            k = index - n // 2
        else:
            k = np.where(index < (n + 1) // 2, index, index - n)
        out[:, a] = k
    return out


def direct_type1(points, strengths, n_modes, isign=1, order=0, select=None, device="cuda:0"):
    """Type-1 FP64 direct sums at the storage indices `select` (all modes when
    None); `strengths` (batch, M); returns (batch, count) complex128."""
    d = len(n_modes)
    return _sums(d, isign, mode_vectors(n_modes, order, select), points, strengths, device=device)


def direct_type2(points, coefficients, n_modes, isign=1, order=0, select=None, device="cuda:0"):
    """Type-2 FP64 direct sums at the points `select` (all points when None);
    `coefficients` (batch, N); returns (batch, count) complex128."""
    d = len(n_modes)
    torch = _torch()
    pts = _as_f64(points, device).reshape(-1, d)
    if select is not None:
        pts = pts[torch.as_tensor(np.asarray(select, dtype=np.int64), device=device)]
    n = int(np.prod(n_modes))
    coefficients = _as_c128(coefficients, device).reshape(-1, n)
    return _sums(d, isign, pts, None, coefficients, modes=n_modes, order=order, device=device)


def direct_type3(sources, strengths, targets, isign=1, select=None, device="cuda:0"):
    """Type-3 FP64 direct sums at the targets `select` (all when None)."""
    torch = _torch()
    src = _as_f64(sources, device)
    d = 1 if src.dim() == 1 else src.shape[1]
    tgt = _as_f64(targets, device).reshape(-1, d)
    if select is not None:
        tgt = tgt[torch.as_tensor(np.asarray(select, dtype=np.int64), device=device)]
    return _sums(d, isign, tgt, src.reshape(-1, d), strengths, device=device)
