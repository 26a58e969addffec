"""NumPy host-array plans with the reference's Python interface
(python/wgpu_nufft/_native.pyi:16-202, python/src/lib.rs): `Context`,
`Type1Plan`, `Type2Plan`, `Type3Plan` and `WgpuNufftError`, running the
CUDA plans of this package on the GPU.

Arrays follow the reference's NumPy conventions: points are float32 of shape
(M, d) (or (M,) in 1D) whose column a is the coordinate along mode axis a;
modes are complex64 arrays of shape n_modes in C order (index [k0, k1, ...]
is mode k0 along axis 0); a leading batch axis (B, ...) selects a batch of
1..batch transforms. Inputs are checked as the reference checks them (dtype,
C-contiguity, finite values, coordinates within [-3 pi, 3 pi] or the type-3
bounds, batch capacity) before anything runs. Calls on one plan are
serialized, as the reference's plans lock their state.

Differences: the reference's CPU plans (`CpuType1Plan` and friends) are not
provided: this package has no CPU engine. Type-1 and type-2 plans take 1 to 8
dimensions, type-3 plans 1 to 3.
"""

from __future__ import annotations

import math
import threading

import numpy as np

from . import NufftConfig, NufftError, NufftPlan, NufftType3Config, NufftType3Plan, Precision, _native

__all__ = ["Context", "Type1Plan", "Type2Plan", "Type3Plan", "WgpuNufftError"]


class WgpuNufftError(RuntimeError):
    """A GPU failure (the reference's wgpu_nufft.WgpuNufftError)."""


def _torch():
    import torch

    return torch


class Context:
    """The CUDA device that plans run on (the reference's persistent wgpu device).

    `power_preference` and `force_fallback` are accepted for compatibility;
    a fallback (software) adapter is not available."""

    def __init__(self, power_preference: str = "high-performance", force_fallback: bool = False,
                 device: int | None = None) -> None:
        if power_preference not in ("high-performance", "low-power", "none"):
            raise ValueError("power_preference must be 'high-performance', 'low-power' or 'none'")
        if force_fallback:
            raise WgpuNufftError("no fallback adapter: this library runs on CUDA devices only")
        torch = _torch()
        if not torch.cuda.is_available():
            raise WgpuNufftError("no CUDA device is available")
        self.device = torch.cuda.current_device() if device is None else int(device)
        self._properties = torch.cuda.get_device_properties(self.device)

    @property
    def adapter_name(self) -> str:
        return self._properties.name

    @property
    def backend(self) -> str:
        return "CUDA"

    @property
    def device_type(self) -> str:
        return "DiscreteGpu"

    @property
    def driver(self) -> str:
        return "NVIDIA"

    @property
    def driver_info(self) -> str:
        torch = _torch()
        return f"CUDA {torch.version.cuda}, compute capability {self._properties.major}.{self._properties.minor}"


def _c_array(name: str, array, dtype) -> np.ndarray:
    if not isinstance(array, np.ndarray) or array.dtype != dtype:
        raise TypeError(f"{name} must be a numpy.ndarray of dtype {np.dtype(dtype).name}")
    if not array.flags.c_contiguous:
        raise ValueError(f"{name} must be C-contiguous; use numpy.ascontiguousarray")
    return array


def _check_complex(name: str, values: np.ndarray) -> None:
    flat = values.reshape(-1)
    bad = ~(np.isfinite(flat.real) & np.isfinite(flat.imag))
    if bad.any():
        raise ValueError(f"{name} contains a non-finite value at flat index {int(np.argmax(bad))}")


def _point_count(name: str, shape, dimensions: int) -> int:
    if len(shape) == 1 and dimensions == 1:
        return shape[0]
    if len(shape) == 2 and shape[1] == dimensions:
        return shape[0]
    raise ValueError(f"{name} must have shape (M, {dimensions})" + (" or (M,)" if dimensions == 1 else ""))


def _check_type12_points(name: str, points: np.ndarray, dimensions: int) -> int:
    count = _point_count(name, points.shape, dimensions)
    flat = points.reshape(-1)
    bad = ~np.isfinite(flat)
    if bad.any():
        raise ValueError(f"{name} contains a non-finite coordinate at flat index {int(np.argmax(bad))}")
    far = np.abs(flat.astype(np.float64)) > 3.0 * math.pi
    if far.any():
        raise ValueError(f"{name} coordinate at flat index {int(np.argmax(far))} is outside [-3*pi, 3*pi]")
    return count


def _vector_batch(name: str, shape, length: int, capacity: int):
    if len(shape) == 1 and shape[0] == length:
        batch, explicit = 1, False
    elif len(shape) == 2 and shape[1] == length:
        batch, explicit = shape[0], True
    else:
        raise ValueError(f"{name} must have shape ({length},) or (B, {length})")
    if batch == 0 or batch > capacity:
        raise ValueError(f"{name} batch {batch} is outside the plan capacity 1..={capacity}")
    return batch, explicit


def _mode_batch(name: str, shape, n_modes, capacity: int):
    if tuple(shape) == tuple(n_modes):
        return 1, False
    if len(shape) == len(n_modes) + 1 and tuple(shape[1:]) == tuple(n_modes):
        batch = shape[0]
        if 1 <= batch <= capacity:
            return batch, True
        raise ValueError(f"{name} batch {batch} is outside the plan capacity 1..={capacity}")
    raise ValueError(f"{name} must have shape {list(n_modes)} or (B, {list(n_modes)})")


def _parse_sign(isign: int) -> int:
    if isign not in (-1, 1):
        raise ValueError("isign must be exactly -1 or 1")
    return isign


def _parse_order(mode_order: str) -> int:
    if mode_order == "centered":
        return 0
    if mode_order == "fft":
        return 1
    raise ValueError("mode_order must be 'centered' or 'fft'")


def _core_from_python(modes: np.ndarray, batch: int, n_modes) -> np.ndarray:
    """(B,) + n_modes in C order -> (B, N) with axis 0 fastest (the plans' order)."""
    d = len(n_modes)
    arranged = modes.reshape((batch,) + tuple(n_modes)).transpose((0,) + tuple(range(d, 0, -1)))
    return np.ascontiguousarray(arranged).reshape(batch, -1)


def _python_from_core(values: np.ndarray, batch: int, n_modes) -> np.ndarray:
    d = len(n_modes)
    arranged = values.reshape((batch,) + tuple(reversed(n_modes))).transpose((0,) + tuple(range(d, 0, -1)))
    return np.ascontiguousarray(arranged)


class _Type12:
    _kind = 1

    def __init__(self, context: Context, n_modes, eps: float = 1.0e-6, isign: int = 1,
                 mode_order: str = "centered", batch: int = 1) -> None:
        n_modes = [int(n) for n in n_modes]
        if any(n < 0 for n in n_modes):
            raise ValueError("mode counts must not be negative")
        self._sign = _parse_sign(isign)
        order = _parse_order(mode_order)
        if batch < 1:
            raise ValueError("invalid NUFFT plan: batch must be at least one")
        self._context = context
        self._n_modes = n_modes
        self._eps = float(eps)
        self._order = mode_order
        self._batch = int(batch)
        self._mode_count = math.prod(n_modes)
        self._lock = threading.Lock()
        config = NufftConfig(tuple(n_modes), eps, isign=self._sign, mode_order=order, batch=batch,
                             precision=Precision.F32)
        try:
            self._plan = NufftPlan(self._kind, config, device=context.device)
        except NufftError as error:
            if error.code in (19, 26, 27, 28):
                raise WgpuNufftError(f"GPU plan creation failed: {error}") from error
            raise ValueError(f"invalid NUFFT plan: {error}") from error

    @property
    def n_modes(self) -> list[int]:
        return list(self._n_modes)

    @property
    def dimensions(self) -> int:
        return len(self._n_modes)

    @property
    def eps(self) -> float:
        return self._eps

    @property
    def isign(self) -> int:
        return self._sign

    @property
    def mode_order(self) -> str:
        return self._order

    @property
    def batch_capacity(self) -> int:
        return self._batch

    def _run(self, points: np.ndarray, inputs: np.ndarray, batch: int, out_len: int) -> np.ndarray:
        torch = _torch()
        dev = f"cuda:{self._context.device}"
        with self._lock:
            try:
                p = torch.from_numpy(points).to(dev)
                x = torch.from_numpy(inputs.view(np.float32)).to(dev).view(torch.complex64)
                out = torch.empty((batch, out_len), dtype=torch.complex64, device=dev)
                self._plan.set_points_gpu(p)
                self._plan.execute_gpu_batch(batch, x, out)
                self._plan.synchronize()
                return out.cpu().numpy()
            except NufftError as error:
                raise WgpuNufftError(str(error)) from error


class Type1Plan(_Type12):
    """Reusable f32 type-1 NUFFT plan."""

    _kind = 1

    def execute(self, points: np.ndarray, strengths: np.ndarray) -> np.ndarray:
        """Type-1 transform: points (M, d) float32 (or (M,) in 1D), strengths
        (M,) or (B, M) complex64; returns the modes in NumPy axis order,
        shape n_modes or (B, *n_modes)."""
        points = _c_array("points", points, np.float32)
        count = _check_type12_points("points", points, self.dimensions)
        strengths = _c_array("strengths", strengths, np.complex64)
        _check_complex("strengths", strengths)
        batch, explicit = _vector_batch("strengths", strengths.shape, count, self._batch)
        shape = ((batch,) if explicit else ()) + tuple(self._n_modes)
        if count == 0:
            return np.zeros(shape, dtype=np.complex64)
        core = self._run(points, strengths.reshape(batch, count), batch, self._mode_count)
        return _python_from_core(core, batch, self._n_modes).reshape(shape)


class Type2Plan(_Type12):
    """Reusable f32 type-2 NUFFT plan."""

    _kind = 2

    def execute(self, points: np.ndarray, coefficients: np.ndarray) -> np.ndarray:
        """Type-2 transform: points (M, d) float32 (or (M,) in 1D),
        coefficients of shape n_modes or (B, *n_modes) complex64 in NumPy axis
        order; returns the values at the points, shape (M,) or (B, M)."""
        points = _c_array("points", points, np.float32)
        count = _check_type12_points("points", points, self.dimensions)
        coefficients = _c_array("coefficients", coefficients, np.complex64)
        _check_complex("coefficients", coefficients)
        batch, explicit = _mode_batch("coefficients", coefficients.shape, self._n_modes, self._batch)
        shape = (batch, count) if explicit else (count,)
        if count == 0:
            return np.zeros(shape, dtype=np.complex64)
        core = _core_from_python(coefficients, batch, self._n_modes)
        return self._run(points, core, batch, count).reshape(shape)


def _bounds(name: str, values) -> list[tuple[float, float]]:
    array = np.asarray(values, dtype=np.float64)
    if array.ndim != 2 or array.shape[1] != 2:
        raise ValueError(f"{name} must have shape (d, 2)")
    out = []
    for axis, (lower, upper) in enumerate(array):
        if not (np.isfinite(lower) and np.isfinite(upper)):
            raise ValueError(f"{name} axis {axis} endpoints must be finite")
        if lower > upper:
            raise ValueError(f"{name} axis {axis} lower endpoint exceeds its upper endpoint")
        out.append((float(lower), float(upper)))
    return out


class Type3Plan:
    """Reusable f32 type-3 NUFFT plan with fixed coordinate bounds."""

    def __init__(self, context: Context, source_bounds, target_bounds, eps: float = 1.0e-6,
                 isign: int = 1, batch: int = 1) -> None:
        self._sources = _bounds("source_bounds", source_bounds)
        self._targets = _bounds("target_bounds", target_bounds)
        if len(self._sources) != len(self._targets):
            raise ValueError("source_bounds and target_bounds must have the same dimension")
        self._sign = _parse_sign(isign)
        if batch < 1:
            raise ValueError("invalid type-3 plan: batch must be at least one")
        self._context = context
        self._eps = float(eps)
        self._batch = int(batch)
        self._lock = threading.Lock()
        config = NufftType3Config(tuple(self._sources), tuple(self._targets), eps=eps, isign=self._sign,
                                  batch=batch, precision=Precision.F32)
        try:
            self._plan = NufftType3Plan(config, device=context.device)
        except NufftError as error:
            raise ValueError(f"invalid type-3 plan: {error}") from error

    @property
    def dimensions(self) -> int:
        return len(self._sources)

    @property
    def source_bounds(self) -> list[tuple[float, float]]:
        return list(self._sources)

    @property
    def target_bounds(self) -> list[tuple[float, float]]:
        return list(self._targets)

    @property
    def outer_grid_shape(self) -> list[int]:
        info = self._plan.info()
        return [int(info.outer_shape[a]) for a in range(self.dimensions)]

    @property
    def eps(self) -> float:
        return self._eps

    @property
    def isign(self) -> int:
        return self._sign

    @property
    def batch_capacity(self) -> int:
        return self._batch

    def _points(self, name: str, points: np.ndarray, bounds) -> int:
        points = _c_array(name, points, np.float32)
        d = len(bounds)
        count = _point_count(name, points.shape, d)
        pts = points.reshape(count, d).astype(np.float64)
        for index in range(count):
            for axis in range(d):
                value = pts[index, axis]
                lower, upper = bounds[axis]
                if not np.isfinite(value):
                    raise ValueError(f"{name} contains a non-finite coordinate at point {index}, axis {axis}")
                if value < lower or value > upper:
                    raise ValueError(f"{name} coordinate at point {index}, axis {axis} is outside "
                                     f"[{lower}, {upper}]")
        return count

    def execute(self, source_points: np.ndarray, strengths: np.ndarray, target_points: np.ndarray) -> np.ndarray:
        """Type-3 transform from source_points (M, d) float32 with strengths
        (M,) or (B, M) complex64 to target_points (N, d) float32, inside the
        plan's bounds; returns (N,) or (B, N) complex64."""
        m = self._points("source_points", source_points, self._sources)
        n = self._points("target_points", target_points, self._targets)
        strengths = _c_array("strengths", strengths, np.complex64)
        _check_complex("strengths", strengths)
        batch, explicit = _vector_batch("strengths", strengths.shape, m, self._batch)
        shape = (batch, n) if explicit else (n,)
        if m == 0 or n == 0:
            return np.zeros(shape, dtype=np.complex64)
        torch = _torch()
        dev = f"cuda:{self._context.device}"
        with self._lock:
            try:
                src = torch.from_numpy(source_points).to(dev)
                tgt = torch.from_numpy(target_points).to(dev)
                c = torch.from_numpy(strengths.reshape(batch, m).view(np.float32)).to(dev).view(torch.complex64)
                out = torch.empty((batch, n), dtype=torch.complex64, device=dev)
                self._plan.encode_gpu_batch(batch, src, c, tgt, out)
                torch.cuda.synchronize(dev)
                return out.cpu().numpy().reshape(shape)
            except NufftError as error:
                raise WgpuNufftError(str(error)) from error


__version__ = _native.library().wgpu_nufft_version().decode() if _native.LIBRARY_PATH.exists() else "0.3.2"
