"""B200-native NUFFT plans with the interface of wgpuNUFFT's NufftPlan.

`NufftConfig` mirrors the reference's builder (src/config.rs:66-229) and
`NufftPlan` its GPU plan (src/plan.rs:403-1229): points, strengths and modes
are torch CUDA tensors in the reference's layouts (point-major coordinates,
interleaved complex values as complex64 / complex128 tensors, modes axis-0
fastest, batches transform-major), and executions are ordered on the current
torch CUDA stream, which plays the part of the reference's command encoder.
All computation runs in libb200nufft.so; nothing here computes a transform.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field, replace

from . import _native

__all__ = [
    "NufftError",
    "NufftConfig",
    "NufftPlan",
    "NufftType3Config",
    "NufftType3Plan",
    "Precision",
    "ModeOrder",
    "SpreadMethod",
    "NufftSign",
    "launch_count",
    "NufftBatch",
    "version",
]

DEFAULT_EPS = 1.0e-6
DEFAULT_SIGMA = 2.0
MAX_NUFFT_DIMENSIONS = 8
MAX_GPU_DIMENSIONS = 3

STATUS_NAMES = {
    0: "Success",
    1: "InvalidBatch",
    2: "InvalidDimensions",
    3: "ZeroMode",
    4: "InvalidTolerance",
    5: "InvalidSigma",
    6: "KernelWidthUnsupported",
    7: "F32ToleranceUnreachable",
    8: "InvalidKernelWidth",
    9: "PrecisionUnsupported",
    10: "InvalidType3Interval",
    11: "Type3GridSizeUnsupported",
    12: "Type3RescalingUnsupported",
    13: "LengthOverflow",
    14: "InputLength",
    15: "FineGridMustBeEven",
    16: "FineGridTooLarge",
    17: "FftShapeUnsupported",
    18: "GpuDimensionsUnsupported",
    19: "GpuExecutionUnavailable",
    20: "GpuDeviceMismatch",
    21: "GpuBufferAliasUnsupported",
    22: "GpuFineGridIndexUnsupported",
    23: "FftExecutionFailed",
    24: "InvalidKernelFourierCoefficient",
    25: "InvalidArgument",
    26: "DeviceError",
    27: "DeviceAllocationFailed",
    28: "DeviceTimeout",
    29: "Internal",
}


class NufftError(Exception):
    """A failure reported by the library; `kind` names the NufftError variant."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.kind = STATUS_NAMES.get(code, f"Status{code}")
        super().__init__(f"{self.kind}: {message}")


def _check(status: int) -> None:
    if status != 0:
        message = _native.library().b200nufft_last_error()
        raise NufftError(status, message.decode() if message else "")


class Precision:
    """FftPrecision, numbered as the reference's C interface numbers it."""

    F64 = 1
    DF64 = 2
    F32 = 3


class ModeOrder:
    CENTERED = 0
    FFT = 1


class SpreadMethod:
    """Type-1 spreading engine (B200NUFFT_SPREAD_*)."""

    AUTO = 0
    CUDA_CORES = 1
    TENSOR_CORES = 2


class NufftSign:
    POSITIVE = 1
    NEGATIVE = -1


@dataclass(frozen=True)
class NufftConfig:
    """NufftConfig: modes per axis, tolerance, sign, order, sigma, batch, precision."""

    n_modes: tuple
    eps: float = DEFAULT_EPS
    isign: int = 1
    mode_order: int = ModeOrder.CENTERED
    sigma: float = DEFAULT_SIGMA
    batch: int = 1
    precision: int = Precision.F32
    spread_method: int = 0

    def __init__(self, n_modes, eps: float = DEFAULT_EPS, *, isign: int = 1,
                 mode_order: int = ModeOrder.CENTERED, sigma: float = DEFAULT_SIGMA,
                 batch: int = 1, precision: int = Precision.F32, spread_method: int = 0):
        object.__setattr__(self, "n_modes", tuple(int(n) for n in n_modes))
        object.__setattr__(self, "eps", float(eps))
        object.__setattr__(self, "isign", 1 if isign >= 0 else -1)
        object.__setattr__(self, "mode_order", int(mode_order))
        object.__setattr__(self, "sigma", float(sigma))
        object.__setattr__(self, "batch", int(batch))
        object.__setattr__(self, "precision", int(precision))
        object.__setattr__(self, "spread_method", int(spread_method))

    # Builder methods of src/config.rs:91-130.
    def with_isign(self, isign: int) -> "NufftConfig":
        return replace(self, isign=1 if isign >= 0 else -1)

    def with_sign(self, sign: int) -> "NufftConfig":
        return self.with_isign(sign)

    def with_mode_order(self, order: int) -> "NufftConfig":
        return replace(self, mode_order=int(order))

    with_modeord = with_mode_order

    def with_sigma(self, sigma: float) -> "NufftConfig":
        return replace(self, sigma=float(sigma))

    def with_batch(self, batch: int) -> "NufftConfig":
        return replace(self, batch=int(batch))

    def with_precision(self, precision: int) -> "NufftConfig":
        return replace(self, precision=int(precision))

    def with_spread_method(self, method: int) -> "NufftConfig":
        """SpreadMethod.AUTO, CUDA_CORES or TENSOR_CORES (no counterpart in the reference)."""
        return replace(self, spread_method=int(method))

    @property
    def dimensions(self) -> int:
        return len(self.n_modes)

    def mode_count(self) -> int:
        count = 1
        for n in self.n_modes:
            count *= n
        return count

    def modeord(self) -> int:
        return self.mode_order

    def _struct(self, kind: int, device: int) -> _native.Config:
        c = _native.Config()
        _native.library().b200nufft_default_config(ctypes.byref(c))
        c.type = kind
        c.dimensions = self.dimensions
        for axis, n in enumerate(self.n_modes[:8]):
            c.n_modes[axis] = n
        c.batch = self.batch
        c.eps = self.eps
        c.isign = self.isign
        c.mode_order = self.mode_order
        c.sigma = self.sigma
        c.precision = self.precision
        c.device = device
        c.spread_method = self.spread_method
        return c


def _torch():
    import torch

    return torch


def _stream_handle(stream) -> int:
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream)


def _nbytes(tensor) -> int:
    return int(tensor.numel()) * int(tensor.element_size())


def _require_bytes(tensor, needed: int, what: str) -> None:
    """The device-pointer interface cannot see buffer sizes; tensors can. A
    tensor smaller than the plan needs is rejected here instead of being
    read or written past its end (the reference validates its buffer sizes
    the same way, src/plan.rs:1311-1387)."""
    if needed > 0 and (tensor is None or _nbytes(tensor) < needed):
        have = 0 if tensor is None else _nbytes(tensor)
        raise NufftError(25, f"{what} holds {have} bytes; the plan needs {needed}")


def _ptr(tensor) -> int:
    if tensor is None:
        return 0
    if not tensor.is_cuda:
        raise NufftError(25, "tensors must live on a CUDA device")
    if not tensor.is_contiguous():
        raise NufftError(25, "tensors must be contiguous")
    return int(tensor.data_ptr())


class NufftPlan:
    """A type-1 or type-2 GPU plan (NufftPlan::type1_gpu / type2_gpu)."""

    def __init__(self, kind: int, config: NufftConfig, device: int | None = None):
        torch = _torch()
        if device is None:
            device = torch.cuda.current_device() if torch.cuda.is_available() else -1
        self.kind = kind
        self.config = config
        self.device = device
        self._handle = ctypes.c_void_p()
        self._points = None
        c = config._struct(kind, device)
        _check(_native.library().b200nufft_plan_create(ctypes.byref(c), ctypes.byref(self._handle)))

    @classmethod
    def type1_gpu(cls, config: NufftConfig, device: int | None = None) -> "NufftPlan":
        return cls(1, config, device)

    @classmethod
    def type2_gpu(cls, config: NufftConfig, device: int | None = None) -> "NufftPlan":
        return cls(2, config, device)

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle and _native is not None:  # module globals are gone at interpreter exit
            _native.library().b200nufft_plan_destroy(handle)
            self._handle = None

    # -- metadata ---------------------------------------------------------
    def info(self) -> _native.PlanInfo:
        info = _native.PlanInfo()
        _check(_native.library().b200nufft_plan_get_info(self._handle, ctypes.byref(info)))
        return info

    def kernel_width(self) -> int:
        return self.info().kernel_width

    def kernel_beta(self) -> float:
        return self.info().kernel_beta

    def fine_grid_shape(self) -> tuple:
        info = self.info()
        return tuple(info.fine_shape[a] for a in range(info.dimensions))

    def bin_geometries(self) -> list:
        info = self.info()
        return [tuple(info.geometry_sides[g][a] for a in range(info.dimensions))
                for g in range(info.geometry_count)]

    def centered_kernel_fourier_coefficients(self, axis: int) -> list:
        count = ctypes.c_int64()
        lib = _native.library()
        _check(lib.b200nufft_plan_kernel_fourier_coefficients(self._handle, axis, None, 0, ctypes.byref(count)))
        values = (ctypes.c_double * count.value)()
        _check(lib.b200nufft_plan_kernel_fourier_coefficients(self._handle, axis, values, count.value, ctypes.byref(count)))
        return list(values)

    # -- buffer sizes (src/plan.rs:732-794, 1032-1078) --------------------
    def _size(self, fn, *args) -> int:
        out = ctypes.c_uint64()
        _check(fn(self._handle, *args, ctypes.byref(out)))
        return out.value

    def required_point_buffer_size_bytes(self, point_count: int) -> int:
        return self._size(_native.library().b200nufft_required_point_bytes, point_count)

    def required_input_buffer_size_bytes(self, point_count: int, active_batch: int | None = None) -> int:
        batch = self.config.batch if active_batch is None else active_batch
        return self._size(_native.library().b200nufft_required_input_bytes, point_count, batch)

    def required_output_buffer_size_bytes(self, point_count: int, active_batch: int | None = None) -> int:
        batch = self.config.batch if active_batch is None else active_batch
        return self._size(_native.library().b200nufft_required_output_bytes, point_count, batch)

    # -- execution ----------------------------------------------------------
    def set_points_gpu(self, points, point_count: int | None = None, stream=None) -> None:
        """Bins `points` (a CUDA tensor, point-major; Df64 plans: (hi, lo)
        float pairs per coordinate) for repeated executions. Without
        `point_count` the count is the tensor's bytes over the bytes of one
        point in the plan's storage."""
        per_point = self.required_point_buffer_size_bytes(1)
        count = _nbytes(points) // per_point if point_count is None else int(point_count)
        _require_bytes(points, self.required_point_buffer_size_bytes(count), "the point buffer")
        _check(_native.library().b200nufft_set_points(self._handle, count, _ptr(points), _stream_handle(stream)))
        self._points = points
        self._count = count
        self._sizes = {}

    def _io_sizes(self, active_batch: int):
        """(input bytes, output bytes) of an execution on the current points."""
        sizes = self._sizes.get(active_batch)
        if sizes is None:
            sizes = (self.required_input_buffer_size_bytes(self._count, active_batch),
                     self.required_output_buffer_size_bytes(self._count, active_batch))
            self._sizes[active_batch] = sizes
        return sizes

    def execute_gpu_batch(self, active_batch: int, inputs, output, stream=None) -> None:
        count = getattr(self, "_count", None)
        if count is not None and 0 < active_batch <= self.config.batch:
            sizes = self._io_sizes(active_batch)
            _require_bytes(inputs, sizes[0], "the input buffer")
            _require_bytes(output, sizes[1], "the output buffer")
        _check(_native.library().b200nufft_execute(self._handle, active_batch, _ptr(inputs), _ptr(output),
                                                   _stream_handle(stream)))

    def execute_gpu(self, inputs, output, stream=None) -> None:
        self.execute_gpu_batch(self.config.batch, inputs, output, stream)

    def encode_gpu_batch(self, active_batch: int, points, inputs, output, stream=None) -> None:
        self.set_points_gpu(points, stream=stream)
        self.execute_gpu_batch(active_batch, inputs, output, stream)

    def encode_gpu(self, points, inputs, output, stream=None) -> None:
        self.encode_gpu_batch(self.config.batch, points, inputs, output, stream)

    # Reference method names.
    def execute_type1_gpu(self, strengths, output, stream=None):
        self._require(1)
        self.execute_gpu(strengths, output, stream)

    def execute_type1_gpu_batch(self, active_batch, strengths, output, stream=None):
        self._require(1)
        self.execute_gpu_batch(active_batch, strengths, output, stream)

    def encode_type1_gpu(self, points, strengths, output, stream=None):
        self._require(1)
        self.encode_gpu(points, strengths, output, stream)

    def encode_type1_gpu_batch(self, active_batch, points, strengths, output, stream=None):
        self._require(1)
        self.encode_gpu_batch(active_batch, points, strengths, output, stream)

    def execute_type2_gpu(self, coefficients, output, stream=None):
        self._require(2)
        self.execute_gpu(coefficients, output, stream)

    def execute_type2_gpu_batch(self, active_batch, coefficients, output, stream=None):
        self._require(2)
        self.execute_gpu_batch(active_batch, coefficients, output, stream)

    def encode_type2_gpu(self, points, coefficients, output, stream=None):
        self._require(2)
        self.encode_gpu(points, coefficients, output, stream)

    def encode_type2_gpu_batch(self, active_batch, points, coefficients, output, stream=None):
        self._require(2)
        self.encode_gpu_batch(active_batch, points, coefficients, output, stream)

    def _require(self, kind: int) -> None:
        if self.kind != kind:
            other = "type-2" if self.kind == 2 else "type-1"
            raise NufftError(19, f"the plan was built for {other} execution")

    def synchronize(self, stream=None) -> None:
        _check(_native.library().b200nufft_plan_synchronize(self._handle, _stream_handle(stream)))

    # -- stage timing (the reference's gpu-profiling stage layout) ---------
    def stage_timing(self, enable: bool = True) -> None:
        """Records CUDA events around every stage of later set_points / execute calls."""
        _check(_native.library().b200nufft_plan_stage_timing(self._handle, 1 if enable else 0))

    def stage_report(self) -> dict:
        """{stage: (milliseconds, launches)} summed since the last report; the caller
        must have synchronized the streams the stages ran on."""
        report = _native.StageReport()
        _check(_native.library().b200nufft_plan_stage_report(self._handle, ctypes.byref(report)))
        return {name: (report.milliseconds[i], report.launches[i])
                for i, name in enumerate(_native.STAGE_NAMES) if report.launches[i]}

    # -- parity hooks -----------------------------------------------------
    def bin_order(self, stream=None):
        """(permutation, bin_offsets) of the last point set, as int64 CPU tensors."""
        torch = _torch()
        info = self.info()
        perm = torch.empty(max(info.point_count, 1), dtype=torch.int32, device=f"cuda:{self.device}")
        offsets = torch.empty(info.bin_count + 1, dtype=torch.int32, device=f"cuda:{self.device}")
        _check(_native.library().b200nufft_copy_bin_order(self._handle, _ptr(perm), _ptr(offsets),
                                                          _stream_handle(stream)))
        self.synchronize(stream)
        mask = (1 << 32) - 1
        return ((perm[: info.point_count].cpu().to(torch.int64) & mask),
                (offsets.cpu().to(torch.int64) & mask))

    def prepared_slots(self, stream=None):
        """(starts, offsets) of the reference's prepared layout for the last point set."""
        torch = _torch()
        info = self.info()
        d = info.dimensions
        n = max(info.point_count, 1)
        starts = torch.empty(n * (d + 1), dtype=torch.int32, device=f"cuda:{self.device}")
        offsets = torch.empty(n * d * 2, dtype=torch.float32, device=f"cuda:{self.device}")
        _check(_native.library().b200nufft_copy_prepared_slots(self._handle, _ptr(starts), _ptr(offsets),
                                                              _stream_handle(stream)))
        self.synchronize(stream)
        return starts[: info.point_count * (d + 1)].cpu(), offsets[: info.point_count * d * 2].cpu()


@dataclass(frozen=True)
class NufftType3Config:
    """NufftType3Config (src/type3.rs:100-213): source and target intervals per axis."""

    source_bounds: tuple
    target_bounds: tuple
    eps: float = 1.0e-9
    isign: int = 1
    sigma: float = DEFAULT_SIGMA
    batch: int = 1
    precision: int = Precision.F64

    @property
    def dimensions(self) -> int:
        return len(self.source_bounds)


class NufftType3Plan:
    """A type-3 GPU plan (NufftType3Plan::new_gpu)."""

    def __init__(self, config: NufftType3Config, device: int | None = None):
        torch = _torch()
        if device is None:
            device = torch.cuda.current_device() if torch.cuda.is_available() else -1
        self.config = config
        self.device = device
        c = _native.Type3Config()
        c.dimensions = config.dimensions
        c.batch = config.batch
        c.eps = config.eps
        c.isign = config.isign
        c.sigma = config.sigma
        c.precision = config.precision
        c.device = device
        for axis, (lo, hi) in enumerate(config.source_bounds):
            c.source_lower[axis], c.source_upper[axis] = lo, hi
        for axis, (lo, hi) in enumerate(config.target_bounds):
            c.target_lower[axis], c.target_upper[axis] = lo, hi
        self._handle = ctypes.c_void_p()
        _check(_native.library().b200nufft_type3_plan_create(ctypes.byref(c), ctypes.byref(self._handle)))

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle and _native is not None:  # module globals are gone at interpreter exit
            _native.library().b200nufft_type3_plan_destroy(handle)
            self._handle = None

    def info(self) -> _native.Type3Info:
        info = _native.Type3Info()
        _check(_native.library().b200nufft_type3_get_info(self._handle, ctypes.byref(info)))
        return info

    def _scalar_bytes(self) -> int:
        return 4 if self.config.precision == Precision.F32 else 8

    def set_points_gpu(self, sources, targets, stream=None) -> None:
        """Sources and targets point-major in the plan's storage (Df64: (hi,
        lo) float pairs per coordinate); the counts follow from their bytes."""
        per_point = self.config.dimensions * self._scalar_bytes()
        sources_count, targets_count = _nbytes(sources) // per_point, _nbytes(targets) // per_point
        _check(_native.library().b200nufft_type3_set_points(
            self._handle, sources_count, _ptr(sources), targets_count, _ptr(targets), _stream_handle(stream)))
        self._points = (sources, targets)
        self._counts = (sources_count, targets_count)

    def execute_gpu_batch(self, active_batch: int, strengths, output, stream=None) -> None:
        counts = getattr(self, "_counts", None)
        if counts is not None and 0 < active_batch <= self.config.batch:
            value = 2 * self._scalar_bytes() * active_batch
            _require_bytes(strengths, value * counts[0], "the strength buffer")
            _require_bytes(output, value * counts[1], "the output buffer")
        _check(_native.library().b200nufft_type3_execute(self._handle, active_batch, _ptr(strengths), _ptr(output),
                                                         _stream_handle(stream)))

    def encode_gpu_batch(self, active_batch, sources, strengths, targets, output, stream=None) -> None:
        self.set_points_gpu(sources, targets, stream)
        self.execute_gpu_batch(active_batch, strengths, output, stream)


class NufftBatch:
    """Many independent 2D/3D f32 type-1 plans (one window width, points set)
    executed together: one persistent spreading launch over every problem's
    tile parts, then each problem's fold, FFT and deconvolution on streams
    forked from the caller's (b200nufft_batch_*). Each problem's modes are
    the bits of its own execution."""

    def __init__(self, plans):
        self.plans = list(plans)
        handles = (ctypes.c_void_p * len(self.plans))(*[p._handle.value for p in self.plans])
        self._handle = ctypes.c_void_p()
        _check(_native.library().b200nufft_batch_create(handles, len(self.plans), ctypes.byref(self._handle)))

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle and _native is not None:
            _native.library().b200nufft_batch_destroy(handle)
            self._handle = None

    def execute(self, strengths, outputs, stream=None) -> None:
        """strengths[p], outputs[p]: CUDA tensors of problem p (one vector)."""
        if len(strengths) != len(self.plans) or len(outputs) != len(self.plans):
            raise NufftError(25, "one strength and one output tensor per plan")
        for plan, s, o in zip(self.plans, strengths, outputs):
            if getattr(plan, "_count", None) is None:
                raise NufftError(19, "every plan of a batch needs its points set")
            sizes = plan._io_sizes(1)
            _require_bytes(s, sizes[0], "a strength buffer")
            _require_bytes(o, sizes[1], "an output buffer")
        ins = (ctypes.c_void_p * len(self.plans))(*[_ptr(s) for s in strengths])
        outs = (ctypes.c_void_p * len(self.plans))(*[_ptr(o) for o in outputs])
        _check(_native.library().b200nufft_batch_execute(self._handle, ins, outs, _stream_handle(stream)))


def launch_count() -> int:
    """Kernel launches issued by the library so far in this process."""
    return int(_native.library().b200nufft_launch_count())


def version() -> str:
    return _native.library().b200nufft_version().decode()
