"""The C-ABI library: it loads, exports every declared symbol, and its host-side
plan logic (validation, metadata, layout choice) matches the oracle. No GPU."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import wgpunufft_b200 as w
from wgpunufft_b200 import _native
from oracle import es_kernel, layout

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    names = []
    for header in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        names += re.findall(r"\b((?:b200nufft|wgpu_nufft)\w*)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _native.library()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def host_plan(kind, n_modes, eps, **kw):
    config = w.NufftConfig(n_modes, eps, **kw)
    c = config._struct(kind, -1)
    handle = ctypes.c_void_p()
    status = _native.library().b200nufft_plan_create_host(ctypes.byref(c), ctypes.byref(handle))
    return status, handle


def status_of(kind, n_modes, eps, **kw):
    status, handle = host_plan(kind, n_modes, eps, **kw)
    if status == 0:
        _native.library().b200nufft_plan_destroy(handle)
    return w.STATUS_NAMES[status]


def test_validation_errors_follow_the_reference():
    assert status_of(1, (8,), 0.0) == "InvalidTolerance"
    assert status_of(1, (8,), 1.0) == "InvalidTolerance"
    assert status_of(1, (8,), float("nan")) == "InvalidTolerance"
    assert status_of(1, (8,), 1e-20) == "KernelWidthUnsupported"
    assert status_of(1, (8,), 1e-6, sigma=1.0) == "InvalidSigma"
    assert status_of(1, (8, 0), 1e-6) == "ZeroMode"
    assert status_of(1, (8,), 1e-6, batch=0) == "InvalidBatch"
    assert status_of(1, (), 1e-6) == "InvalidDimensions"
    assert status_of(1, (2,) * 9, 1e-6) == "InvalidDimensions"
    assert status_of(1, (4,) * 4, 1e-6) == "Success"
    assert status_of(2, (3,) * 8, 1e-2) == "Success"
    assert status_of(1, (1000,), 1e-6, sigma=1.0e15) == "FineGridTooLarge"
    # src/config.rs:310-318: sigma 1.25 at 1e-6 misses f32 by far in 2D and 3D.
    assert status_of(1, (256, 256), 1e-6, sigma=1.25) == "F32ToleranceUnreachable"
    assert status_of(2, (64, 64, 64), 1e-6, sigma=1.25) == "F32ToleranceUnreachable"
    assert status_of(1, (1024, 1024), 1e-9) == "Success"
    assert status_of(1, (1 << 23,), 1e-6) == "GpuFineGridIndexUnsupported"


@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("n_modes,eps,sigma", [
    ((17,), 1e-6, 2.0), ((64, 64), 1e-6, 2.0), ((1024, 1024), 1e-5, 2.0), ((256, 256, 256), 1e-5, 2.0),
    ((6, 5), 1e-3, 2.0), ((4, 3, 5), 1e-5, 2.0), ((17, 9), 1e-4, 1.25), ((512, 512), 1e-3, 2.0),
])
def test_plan_metadata_matches_oracle(kind, n_modes, eps, sigma):
    status, handle = host_plan(kind, n_modes, eps, sigma=sigma)
    assert status == 0
    lib = _native.library()
    try:
        info = _native.PlanInfo()
        assert lib.b200nufft_plan_get_info(handle, ctypes.byref(info)) == 0
        width, beta = es_kernel.es_parameters(eps, sigma)
        assert info.kernel_width == width and info.kernel_beta == pytest.approx(beta, abs=1e-13)
        fine = [es_kernel.select_fine_grid_size(n, sigma, width) for n in n_modes]
        assert list(info.fine_shape[: len(n_modes)]) == fine
        for axis, n in enumerate(fine):
            count = ctypes.c_int64()
            values = (ctypes.c_double * (n // 2 + 1))()
            assert lib.b200nufft_plan_kernel_fourier_coefficients(handle, axis, values, n // 2 + 1, ctypes.byref(count)) == 0
            expected = es_kernel.centered_fourier_coefficients(width, beta, n)
            np.testing.assert_allclose(np.array(values), expected, rtol=1e-13, atol=1e-15)
        lay = layout.Layout(width, fine, "F32")
        sides = [list(info.geometry_sides[g][: len(n_modes)]) for g in range(info.geometry_count)]
        assert sides == [g.side for g in lay.geometries]
        if kind == 1:
            for m in [0, 1, 100, 10_000, 1_000_000, 10_000_000, 50_000_000]:
                g = ctypes.c_int32()
                assert lib.b200nufft_plan_choose_geometry(handle, m, ctypes.byref(g)) == 0
                assert g.value == lay.choose_geometry(m), m
        size = ctypes.c_uint64()
        assert lib.b200nufft_required_point_bytes(handle, 1000, ctypes.byref(size)) == 0
        assert size.value == 1000 * len(n_modes) * 4
        assert lib.b200nufft_required_input_bytes(handle, 1000, 1, ctypes.byref(size)) == 0
        n_total = int(np.prod(n_modes))
        assert size.value == (1000 if kind == 1 else n_total) * 8
        status = lib.b200nufft_required_output_bytes(handle, 1000, 2, ctypes.byref(size))
        assert w.STATUS_NAMES[status] == "InvalidBatch"
        status = lib.b200nufft_set_points(handle, 10, None, None)
        assert w.STATUS_NAMES[status] == "GpuExecutionUnavailable"
    finally:
        lib.b200nufft_plan_destroy(handle)


@pytest.mark.parametrize("shape,eps", [
    ([128], 1e-6), ([14], 1e-6), ([4096], 1e-3), ([36, 36], 1e-6), ([2000, 2000], 1e-6), ([2048, 2048], 1e-5),
    ([200, 200, 200], 1e-6), ([400, 400, 400], 1e-6), ([512, 512, 512], 1e-5), ([64, 32, 16], 1e-9),
    ([1080, 1080, 1080], 1e-9), ([24, 30, 18], 1e-12),
])
def test_cpp_layout_matches_oracle_layout(shape, eps):
    """The library's restatement of for_grid / choose_geometry agrees with the
    oracle's, which the known answers pin."""
    width = es_kernel.es_parameters(eps, 2.0)[0]
    n_modes = [s // 2 for s in shape]
    status, handle = host_plan(1, n_modes, eps)
    assert status == 0
    lib = _native.library()
    try:
        info = _native.PlanInfo()
        lib.b200nufft_plan_get_info(handle, ctypes.byref(info))
        fine = list(info.fine_shape[: len(shape)])
        lay = layout.Layout(width, fine, "F32")
        sides = [list(info.geometry_sides[g][: len(shape)]) for g in range(info.geometry_count)]
        assert sides == [g.side for g in lay.geometries]
        for m in [1, 50, 3_000, 250_000, 4_000_000, 70_000_000]:
            g = ctypes.c_int32()
            lib.b200nufft_plan_choose_geometry(handle, m, ctypes.byref(g))
            assert g.value == lay.choose_geometry(m)
    finally:
        lib.b200nufft_plan_destroy(handle)


def test_tuning_lookup_is_frozen_per_key_and_override_validates():
    """The tuning table gives one answer per workload key (so outputs repeat
    bit for bit); the tuner's override replaces only its non-zero fields and
    rejects tile sides that are not powers of two."""
    from wgpunufft_b200 import _native

    lib = _native.library()

    def lookup(*key):
        out = _native.Tuning()
        assert lib.b200nufft_tuning_lookup(*key, ctypes.byref(out)) == 0
        return (out.tile, out.ctas_per_sm, out.crowded_ctas_per_sm, out.tensor_min_batch)

    key = (1, 2, 3, 6, 2048 * 2048, 10_000_000)
    first = lookup(*key)
    assert lookup(*key) == first
    assert first[1] >= 1 and first[2] >= 1 and first[3] >= 1
    assert lib.b200nufft_tuning_override(_native.Tuning(32, 0, 0, 0)) == 0
    try:
        overridden = lookup(*key)
        assert overridden[0] == 32 and overridden[1:] == first[1:]
    finally:
        assert lib.b200nufft_tuning_override(None) == 0
    assert lookup(*key) == first
    assert lib.b200nufft_tuning_override(_native.Tuning(48, 0, 0, 0)) == 25
    assert lookup(*key) == first
