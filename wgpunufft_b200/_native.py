"""ctypes declarations of libb200nufft.so (include/b200_nufft.h, include/wgpu_nufft.h).

The library is loaded from this package directory only; a missing or stale
build raises instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIBRARY_PATH = Path(__file__).resolve().parent / "libb200nufft.so"

c_int = ctypes.c_int
c_int32 = ctypes.c_int32
c_int64 = ctypes.c_int64
c_uint64 = ctypes.c_uint64
c_double = ctypes.c_double
c_float = ctypes.c_float
c_void_p = ctypes.c_void_p
c_char_p = ctypes.c_char_p


class Config(ctypes.Structure):
    _fields_ = [
        ("type", c_int32),
        ("dimensions", c_int32),
        ("n_modes", c_int64 * 8),
        ("batch", c_int64),
        ("eps", c_double),
        ("isign", c_int32),
        ("mode_order", c_int32),
        ("sigma", c_double),
        ("precision", c_int32),
        ("device", c_int32),
        ("spread_method", c_int32),
    ]


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("type", c_int32),
        ("dimensions", c_int32),
        ("precision", c_int32),
        ("kernel_width", c_int32),
        ("kernel_beta", c_double),
        ("fine_shape", c_int64 * 8),
        ("mode_count", c_int64),
        ("batch", c_int64),
        ("geometry_count", c_int32),
        ("geometry_sides", (c_int32 * 8) * 16),
        ("point_count", c_int64),
        ("chosen_geometry", c_int32),
        ("bin_count", c_int64),
    ]


STAGE_NAMES = ("bin_keys", "digit_scan", "radix_passes", "bin_offsets", "tile_parts", "strength_scale",
               "spread", "fold", "fft", "deconvolution", "predeconvolution", "interpolation")


class StageReport(ctypes.Structure):
    _fields_ = [("milliseconds", c_double * 12), ("launches", c_int64 * 12)]


class Type3Config(ctypes.Structure):
    _fields_ = [
        ("dimensions", c_int32),
        ("batch", c_int64),
        ("eps", c_double),
        ("isign", c_int32),
        ("sigma", c_double),
        ("precision", c_int32),
        ("device", c_int32),
        ("source_lower", c_double * 8),
        ("source_upper", c_double * 8),
        ("target_lower", c_double * 8),
        ("target_upper", c_double * 8),
    ]


class Type3Info(ctypes.Structure):
    _fields_ = [
        ("dimensions", c_int32),
        ("kernel_width", c_int32),
        ("kernel_beta", c_double),
        ("outer_shape", c_int64 * 8),
        ("inner_fine_shape", c_int64 * 8),
        ("source_center", c_double * 8),
        ("target_center", c_double * 8),
        ("gamma", c_double * 8),
        ("h", c_double * 8),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [
        ("tile", c_int32),
        ("ctas_per_sm", c_int32),
        ("crowded_ctas_per_sm", c_int32),
        ("tensor_min_batch", c_int32),
    ]


class WgpuOpts(ctypes.Structure):
    _fields_ = [
        ("backend", c_int32),
        ("precision", c_int32),
        ("mode_order", c_int32),
        ("threads", c_int32),
        ("sigma", c_double),
        ("adapter_index", c_int32),
        ("adapter_name", ctypes.c_char * 256),
        ("adapter_pci_bus_id", ctypes.c_char * 32),
    ]


# Every symbol include/b200_nufft.h and include/wgpu_nufft.h declare, with
# its (restype, argtypes). Tests check that the library exports them all.
PLAN = c_void_p
P = ctypes.POINTER
SIGNATURES: dict[str, tuple] = {
    # b200_nufft.h
    "b200nufft_default_config": (None, [P(Config)]),
    "b200nufft_plan_create": (c_int, [P(Config), P(PLAN)]),
    "b200nufft_plan_create_host": (c_int, [P(Config), P(PLAN)]),
    "b200nufft_plan_choose_geometry": (c_int, [PLAN, c_int64, P(c_int32)]),
    "b200nufft_plan_destroy": (None, [PLAN]),
    "b200nufft_plan_get_info": (c_int, [PLAN, P(PlanInfo)]),
    "b200nufft_plan_kernel_fourier_coefficients": (c_int, [PLAN, c_int32, P(c_double), c_int64, P(c_int64)]),
    "b200nufft_required_point_bytes": (c_int, [PLAN, c_int64, P(c_uint64)]),
    "b200nufft_required_input_bytes": (c_int, [PLAN, c_int64, c_int64, P(c_uint64)]),
    "b200nufft_required_output_bytes": (c_int, [PLAN, c_int64, c_int64, P(c_uint64)]),
    "b200nufft_set_points": (c_int, [PLAN, c_int64, c_void_p, c_void_p]),
    "b200nufft_execute": (c_int, [PLAN, c_int64, c_void_p, c_void_p, c_void_p]),
    "b200nufft_encode": (c_int, [PLAN, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "b200nufft_copy_bin_order": (c_int, [PLAN, c_void_p, c_void_p, c_void_p]),
    "b200nufft_plan_synchronize": (c_int, [PLAN, c_void_p]),
    "b200nufft_copy_prepared_slots": (c_int, [PLAN, c_void_p, c_void_p, c_void_p]),
    "b200nufft_plan_stage_timing": (c_int, [PLAN, c_int32]),
    "b200nufft_plan_stage_report": (c_int, [PLAN, P(StageReport)]),
    "b200nufft_type3_plan_create": (c_int, [P(Type3Config), P(PLAN)]),
    "b200nufft_type3_plan_destroy": (None, [PLAN]),
    "b200nufft_type3_get_info": (c_int, [PLAN, P(Type3Info)]),
    "b200nufft_type3_set_points": (c_int, [PLAN, c_int64, c_void_p, c_int64, c_void_p, c_void_p]),
    "b200nufft_type3_execute": (c_int, [PLAN, c_int64, c_void_p, c_void_p, c_void_p]),
    "b200nufft_bin_order_noalloc": (c_int, [c_int32, P(c_int64), c_int32, P(c_int32), c_int64,
                                            c_void_p, c_void_p, c_void_p, c_void_p]),
    "b200nufft_last_error": (c_char_p, []),
    "b200nufft_version": (c_char_p, []),
    "b200nufft_launch_count": (c_uint64, []),
    "b200nufft_batch_create": (c_int, [P(PLAN), c_int32, P(PLAN)]),
    "b200nufft_batch_destroy": (None, [PLAN]),
    "b200nufft_batch_execute": (c_int, [PLAN, P(c_void_p), P(c_void_p), c_void_p]),
    "b200nufft_tuning_lookup": (c_int, [c_int32, c_int32, c_int32, c_int32, c_int64, c_int64, P(Tuning)]),
    "b200nufft_tuning_override": (c_int, [P(Tuning)]),
    "b200nufft_set_fused_transforms": (c_int, [c_int]),
    "b200nufft_tf32_peak": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_int, P(c_float), P(c_uint64)]),
    # wgpu_nufft.h
    "wgpu_nufft_default_opts": (None, [P(WgpuOpts)]),
    "wgpu_nufft_list_adapters": (c_int, [c_void_p, c_int32, P(c_int32)]),
    "wgpu_nufft_last_error": (c_char_p, []),
    "wgpu_nufft_version": (c_char_p, []),
    "wgpu_nufft_gpu_name": (c_char_p, []),
    "wgpu_nufft_shutdown": (None, []),
    "b200nufft_resolve_adapter": (c_int, [P(c_char_p), P(c_char_p), c_int32, P(WgpuOpts), P(c_int32)]),
}

# The two host-array families differ only in their prefix; array arguments
# are raw addresses (numpy .ctypes.data), so both share the signatures.
_A = c_void_p
_O = P(WgpuOpts)
for _prefix in ("wgpu_nufft", "wgpu_nufftf"):
    SIGNATURES.update({
        f"{_prefix}_makeplan": (c_int, [c_int32, c_int32, P(c_int64), c_int32, c_int64, c_double, P(PLAN), _O]),
        f"{_prefix}_setpts": (c_int, [PLAN, c_int64, _A, _A, _A, c_int64, _A, _A, _A]),
        f"{_prefix}_setpts_nd": (c_int, [PLAN, c_int64, _A, c_int64, _A]),
        f"{_prefix}_execute": (c_int, [PLAN, _A, _A]),
        f"{_prefix}_destroy": (None, [PLAN]),
        f"{_prefix}_plan_backend": (c_int, [PLAN]),
        f"{_prefix}_plan_precision": (c_int, [PLAN]),
        f"{_prefix}1d1": (c_int, [c_int64, _A, _A, c_int32, c_double, c_int64, _A, _O]),
        f"{_prefix}1d2": (c_int, [c_int64, _A, _A, c_int32, c_double, c_int64, _A, _O]),
        f"{_prefix}1d3": (c_int, [c_int64, _A, _A, c_int32, c_double, c_int64, _A, _A, _O]),
        f"{_prefix}2d1": (c_int, [c_int64, _A, _A, _A, c_int32, c_double, c_int64, c_int64, _A, _O]),
        f"{_prefix}2d2": (c_int, [c_int64, _A, _A, _A, c_int32, c_double, c_int64, c_int64, _A, _O]),
        f"{_prefix}2d3": (c_int, [c_int64, _A, _A, _A, c_int32, c_double, c_int64, _A, _A, _A, _O]),
        f"{_prefix}3d1": (c_int, [c_int64, _A, _A, _A, _A, c_int32, c_double, c_int64, c_int64, c_int64, _A, _O]),
        f"{_prefix}3d2": (c_int, [c_int64, _A, _A, _A, _A, c_int32, c_double, c_int64, c_int64, c_int64, _A, _O]),
        f"{_prefix}3d3": (c_int, [c_int64, _A, _A, _A, _A, c_int32, c_double, c_int64, _A, _A, _A, _A, _O]),
    })


class WgpuAdapter(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 256),
        ("backend", ctypes.c_char * 16),
        ("device_type", ctypes.c_char * 16),
        ("pci_bus_id", ctypes.c_char * 32),
        ("is_default", c_int32),
    ]

_lib: ctypes.CDLL | None = None


def library() -> ctypes.CDLL:
    """The loaded CUDA library; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY_PATH.exists():
        raise RuntimeError(
            f"{LIBRARY_PATH} is missing: build it with `python -m wgpunufft_b200.build` "
            "(there is no CPU fallback)"
        )
    lib = ctypes.CDLL(os.fspath(LIBRARY_PATH))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib
