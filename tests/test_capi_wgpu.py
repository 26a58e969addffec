"""The host-array C interface (include/wgpu_nufft.h), following the
reference's capi/tests/c_api.rs: one-call and plan suites against FP64
direct sums, precision options, error codes with their messages, the options
layout, and adapter selection (capi/src/adapter.rs tests, on a fake list).

Tests without the gpu mark call only what needs no device."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import native
from tests.conftest import rel_l2
from wgpunufft_b200 import _native

lib = _native.library()

AUTO, GPU, CPU = 0, 1, 2
P_AUTO, P_F64, P_DF64, P_F32 = 0, 1, 2, 3


def opts(backend=AUTO, precision=P_AUTO, mode_order=0, sigma=0.0, name=b"", pci=b"", index=0):
    o = _native.WgpuOpts()
    lib.wgpu_nufft_default_opts(ctypes.byref(o))
    o.backend, o.precision, o.mode_order, o.sigma = backend, precision, mode_order, sigma
    o.adapter_name, o.adapter_pci_bus_id, o.adapter_index = name, pci, index
    return o


def last_error() -> str:
    return lib.wgpu_nufft_last_error().decode()


def ptr(array):
    return None if array is None else array.ctypes.data


def interleaved(values, dtype=np.float64):
    return np.ascontiguousarray(np.asarray(values).astype(np.complex128)).view(np.float64).astype(dtype)


def complex_of(values):
    return np.asarray(values, dtype=np.float64).view(np.complex128)


def makeplan(kind, n_modes, eps=1e-6, isign=1, ntrans=1, options=None, single=False):
    prefix = "wgpu_nufftf" if single else "wgpu_nufft"
    plan = ctypes.c_void_p()
    modes = (ctypes.c_int64 * max(1, len(n_modes)))(*n_modes)
    dim = len(n_modes) if kind != 3 else n_modes[0]
    code = getattr(lib, f"{prefix}_makeplan")(kind, dim, modes, isign, ntrans, eps, ctypes.byref(plan),
                                               None if options is None else ctypes.byref(options))
    return code, plan


# ---------------------------------------------------------------------------
# No device needed.


def test_options_layout_and_defaults():
    """capi/tests/c_api.rs:510-527: the shared layouts and an all-zero default."""
    assert ctypes.sizeof(_native.WgpuOpts) == 320
    assert _native.WgpuOpts.adapter_index.offset == 24
    assert _native.WgpuOpts.adapter_name.offset == 28
    assert _native.WgpuOpts.adapter_pci_bus_id.offset == 284
    assert ctypes.sizeof(_native.WgpuAdapter) == 324
    o = _native.WgpuOpts()
    o.adapter_index, o.adapter_name, o.sigma = 5, b"NVIDIA B200", 3.0
    lib.wgpu_nufft_default_opts(ctypes.byref(o))
    assert bytes(o) == bytes(ctypes.sizeof(o))
    assert lib.wgpu_nufft_version().decode() == "0.3.2"


def test_errors_before_any_device_are_reported_with_messages():
    """capi/tests/c_api.rs:433-507 for the checks that precede the device."""
    code, plan = makeplan(4, [8])
    assert code == 1 and "type" in last_error() and not plan.value
    assert makeplan(1, [0])[0] == 1
    assert makeplan(1, [8], ntrans=0)[0] == 1
    assert makeplan(1, [8], eps=float("nan"))[0] == 1
    assert makeplan(1, [8], eps=0.0)[0] == 1
    plan = ctypes.c_void_p()
    assert lib.wgpu_nufft_makeplan(1, 0, (ctypes.c_int64 * 1)(8), 1, 1, 1e-6, ctypes.byref(plan), None) == 1
    assert "dim" in last_error()
    assert lib.wgpu_nufft_makeplan(1, 1, None, 1, 1, 1e-6, ctypes.byref(plan), None) == 1
    assert lib.wgpu_nufft_makeplan(1, 1, (ctypes.c_int64 * 1)(8), 1, 1, 1e-6, None, None) == 1
    for bad in (opts(backend=7), opts(precision=9), opts(mode_order=2), opts(sigma=0.5),
                opts(sigma=float("inf"))):
        assert makeplan(1, [8], options=bad)[0] == 1, last_error()
    threads = opts()
    threads.threads = -1
    assert makeplan(1, [8], options=threads)[0] == 1
    negative = opts(index=-1)
    assert makeplan(1, [8], options=negative)[0] == 1 and "adapter_index" in last_error()
    unterminated = opts()
    ctypes.memmove(ctypes.addressof(unterminated) + _native.WgpuOpts.adapter_name.offset, b"a" * 256, 256)
    assert makeplan(1, [8], options=unterminated)[0] == 1 and "adapter_name" in last_error()
    assert makeplan(1, [8], options=opts(pci=b"slot 3"))[0] == 1 and "PCI address" in last_error()
    # No CPU engine: the CPU backend is a plan error, never a fallback.
    code, plan = makeplan(1, [8], options=opts(backend=CPU))
    assert code == 2 and "CPU" in last_error() and not plan.value
    # One-call functions validate the same way.
    x = np.zeros(4)
    c = np.zeros(8)
    f = np.zeros(16)
    assert lib.wgpu_nufft1d1(4, ptr(x), ptr(c), 1, 1e-6, 0, ptr(f), None) == 1
    assert lib.wgpu_nufft1d1(-1, ptr(x), ptr(c), 1, 1e-6, 8, ptr(f), ctypes.byref(opts(backend=CPU))) == 1
    # Null handles.
    lib.wgpu_nufft_destroy(None)
    lib.wgpu_nufftf_destroy(None)
    assert lib.wgpu_nufft_plan_backend(None) == -1
    assert lib.wgpu_nufftf_plan_precision(None) == -1
    assert lib.wgpu_nufft_execute(None, None, None) == 1
    assert lib.wgpu_nufft_setpts(None, 0, None, None, None, 0, None, None, None) == 1


def test_list_adapters_argument_checks():
    count = ctypes.c_int32(-5)
    assert lib.wgpu_nufft_list_adapters(None, 0, None) == 1
    assert lib.wgpu_nufft_list_adapters(None, 1, ctypes.byref(count)) == 1
    assert lib.wgpu_nufft_list_adapters(None, -1, ctypes.byref(count)) == 1
    assert "capacity" in last_error()


def _resolve(entries, **selection):
    names = (ctypes.c_char_p * len(entries))(*[n.encode() for n, _ in entries])
    pcis = (ctypes.c_char_p * len(entries))(*[p.encode() for _, p in entries])
    position = ctypes.c_int32(-9)
    code = lib.b200nufft_resolve_adapter(names, pcis, len(entries), ctypes.byref(opts(**selection)),
                                         ctypes.byref(position))
    return code, position.value


MACHINE = [
    ("Intel UHD", "0000:00:02.0"),
    ("RTX 4090", "0000:01:00.0"),
    ("RTX 4090", "0000:02:00.0"),
    ("Intel UHD", "0000:00:02.0"),
]


def test_adapter_selection_rules():
    """capi/src/adapter.rs:266-340 on a list of this library's kind (each GPU
    listed once)."""
    assert _resolve(MACHINE) == (0, 0)
    assert _resolve(MACHINE, name=b" rtx 4090 ", index=2) == (0, 2)
    assert _resolve(MACHINE, name=b"RTX 4090")[0] == 1
    assert last_error().startswith("2 CUDA adapters match") and "adapter_index" in last_error()
    assert _resolve(MACHINE, name=b"Intel")[0] == 3
    assert "1. Intel UHD" in last_error()
    assert _resolve(MACHINE, pci=b"0000:02:00.0") == (0, 2)
    assert _resolve(MACHINE, pci=b"02:00") == (0, 2)
    assert _resolve(MACHINE, pci=b"00000000:01:00.0") == (0, 1)
    assert _resolve(MACHINE, pci=b" 01:00.0 ") == (0, 1)
    assert _resolve(MACHINE, pci=b"0000:01:00.1")[0] == 3
    assert _resolve(MACHINE, index=1) == (0, 0)
    assert _resolve(MACHINE, index=4) == (0, 3)
    assert _resolve(MACHINE, index=5)[0] == 3 and "index 5" in last_error()
    assert _resolve(MACHINE, name=b"Radeon")[0] == 3
    assert 'name "Radeon"' in last_error() and "2. RTX 4090 (CUDA, DiscreteGpu, 0000:01:00.0)" in last_error()
    assert _resolve([], pci=b"0000:01:00.0")[0] == 3 and last_error().endswith("are none")
    assert _resolve([])[0] == 3
    # A device that reports no address matches no address.
    assert _resolve([("Apple M2", "")], pci=b"0000:00:00.0")[0] == 3
    assert _resolve([("Apple M2", "")], name=b"apple m2") == (0, 0)
    for bad in (b"1", b"0000:01:00.", b"g0:01:00.0", b"0:0:0:0", b"+1:00.0", b"1:2:3:4.0", b"123456789:0:0"):
        assert _resolve(MACHINE, pci=bad)[0] == 1, bad


def test_without_a_device_plans_report_gpu_unavailable():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    code, plan = makeplan(1, [8])
    assert code == 3 and not plan.value
    count = ctypes.c_int32(-1)
    assert lib.wgpu_nufft_list_adapters(None, 0, ctypes.byref(count)) == 0 and count.value == 0
    assert lib.wgpu_nufft_gpu_name().decode() == ""


# ---------------------------------------------------------------------------
# On the GPU.


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _values(rng, count, scale):
    return rng.uniform(-scale, scale, count)


def one_call_suite(precision, eps, tolerance, single=False):
    """capi/tests/c_api.rs:216-296 over all nine one-call functions."""
    rng = np.random.default_rng([0x5EED, precision, int(single)])
    real = np.float32 if single else np.float64
    prefix = "wgpu_nufftf" if single else "wgpu_nufft"
    o = opts(GPU, precision)
    m = 60
    x, y, z = (_values(rng, m, np.pi).astype(real) for _ in range(3))
    c = (rng.standard_normal(m) + 1j * rng.standard_normal(m))
    cr = interleaved(c, real)
    c_used = complex_of(cr.astype(np.float64)) if single else c
    pts = np.stack([x, y, z], axis=1).astype(np.float64)
    isign = -1
    modes = {1: [12], 2: [8, 6], 3: [5, 4, 3]}
    for d in (1, 2, 3):
        axes = [x, y, z][:d]
        n = modes[d]
        count = int(np.prod(n))
        # Type 1.
        f = np.zeros(2 * count, real)
        fn = getattr(lib, f"{prefix}{d}d1")
        assert fn(m, *map(ptr, axes), ptr(cr), isign, eps, *n, ptr(f), ctypes.byref(o)) == 0, last_error()
        ref = native.direct_type1(pts[:, :d], c_used[None], n, isign)[0]
        assert rel_l2(complex_of(f.astype(np.float64)), ref) < tolerance, (d, "type 1")
        # Type 2.
        fm = rng.standard_normal(count) + 1j * rng.standard_normal(count)
        fmr = interleaved(fm, real)
        fm_used = complex_of(fmr.astype(np.float64)) if single else fm
        out = np.zeros(2 * m, real)
        fn = getattr(lib, f"{prefix}{d}d2")
        assert fn(m, *map(ptr, axes), ptr(out), isign, eps, *n, ptr(fmr), ctypes.byref(o)) == 0, last_error()
        ref = native.direct_type2(pts[:, :d], fm_used[None], n, isign)[0]
        assert rel_l2(complex_of(out.astype(np.float64)), ref) < tolerance, (d, "type 2")
        # Type 3.
        nt = 45
        targets = [(_values(rng, nt, 12.0)).astype(real) for _ in range(d)]
        out = np.zeros(2 * nt, real)
        fn = getattr(lib, f"{prefix}{d}d3")
        assert fn(m, *map(ptr, axes), ptr(cr), isign, eps, nt, *map(ptr, targets), ptr(out),
                  ctypes.byref(o)) == 0, last_error()
        ref = native.direct_type3(pts[:, :d], c_used[None], np.stack(targets, 1).astype(np.float64), isign)[0]
        assert rel_l2(complex_of(out.astype(np.float64)), ref) < tolerance, (d, "type 3")


def _fft_order(centered, n_modes):
    """Centered mode array (axis 0 fastest) to FFT order: frequency k at k mod n."""
    shape = tuple(reversed(n_modes))
    grid = np.asarray(centered).reshape(shape)
    return np.fft.ifftshift(grid).reshape(-1)


def plan_suite(precision, eps, tolerance):
    """capi/tests/c_api.rs:298-381: a type-1 plan in FFT order with three
    transforms, points given per axis and then point-major."""
    rng = np.random.default_rng(0xBEEF)
    n_modes = [10, 7]
    count = 70
    ntrans = 3
    code, plan = makeplan(1, n_modes, eps=eps, ntrans=ntrans, options=opts(GPU, precision, mode_order=1))
    assert code == 0, last_error()
    try:
        backend, used = lib.wgpu_nufft_plan_backend(plan), lib.wgpu_nufft_plan_precision(plan)
        for round_ in range(2):
            m = 30 + 11 * round_
            x = _values(rng, m, 3 * np.pi)
            y = _values(rng, m, np.pi)
            c = rng.standard_normal((ntrans, m)) + 1j * rng.standard_normal((ntrans, m))
            if round_ == 0:
                assert lib.wgpu_nufft_setpts(plan, m, ptr(x), ptr(y), None, 0, None, None, None) == 0, last_error()
            else:
                pts = np.ascontiguousarray(np.stack([x, y], 1))
                assert lib.wgpu_nufft_setpts_nd(plan, m, ptr(pts), 0, None) == 0, last_error()
            cr = interleaved(c)
            f = np.zeros(2 * count * ntrans)
            assert lib.wgpu_nufft_execute(plan, ptr(cr), ptr(f)) == 0, last_error()
            got = complex_of(f).reshape(ntrans, count)
            centered = native.direct_type1(np.stack([x, y], 1), c, n_modes, 1)
            for t in range(ntrans):
                assert rel_l2(got[t], _fft_order(centered[t], n_modes)) < tolerance, (round_, t)
        return backend, used
    finally:
        lib.wgpu_nufft_destroy(plan)


@pytest.mark.gpu
def test_gpu_one_call_and_plan_suites_match_direct_sums():
    """capi/tests/c_api.rs:672-700: f64, Df64 and f32 arithmetic on double
    arrays, and the float family."""
    _gpu()
    name = lib.wgpu_nufft_gpu_name().decode()
    assert name.endswith("(CUDA)"), name
    one_call_suite(P_AUTO, 1e-9, 1e-8)
    assert plan_suite(P_AUTO, 1e-9, 1e-8) == (GPU, P_F64)
    one_call_suite(P_DF64, 1e-9, 1e-8)
    assert plan_suite(P_DF64, 1e-9, 1e-8) == (GPU, P_DF64)
    one_call_suite(P_F32, 1e-5, 1e-4)
    assert plan_suite(P_F32, 1e-5, 1e-4) == (GPU, P_F32)
    one_call_suite(P_AUTO, 1e-5, 1e-4, single=True)
    # Repeated one-call transforms reuse their kept plans and stay right.
    one_call_suite(P_AUTO, 1e-9, 1e-8)


@pytest.mark.gpu
def test_gpu_single_precision_plans():
    """capi/tests/c_api.rs:383-421."""
    _gpu()
    rng = np.random.default_rng(0xF32)
    m = 50
    x = _values(rng, m, np.pi).astype(np.float32)
    c = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    cr = interleaved(c, np.float32)
    code, plan = makeplan(2, [16], eps=1e-5, single=True)
    assert code == 0, last_error()
    try:
        assert lib.wgpu_nufftf_plan_precision(plan) == P_F32
        assert lib.wgpu_nufftf_plan_backend(plan) == GPU
        # Type 2 through the plan: 16 modes to 50 points, twice.
        for seed in (1, 2):
            fm = np.random.default_rng(seed).standard_normal(16) + 0j
            fr = interleaved(fm, np.float32)
            assert lib.wgpu_nufftf_setpts(plan, m, ptr(x), None, None, 0, None, None, None) == 0, last_error()
            out = np.zeros(2 * m, np.float32)
            assert lib.wgpu_nufftf_execute(plan, ptr(out), ptr(fr)) == 0, last_error()
            ref = native.direct_type2(x.astype(np.float64)[:, None], fm[None], [16], 1)[0]
            assert rel_l2(complex_of(out.astype(np.float64)), ref) < 1e-4
        # The double functions refuse a float plan.
        assert lib.wgpu_nufft_execute(plan, None, None) == 1 and "array type" in last_error()
    finally:
        lib.wgpu_nufftf_destroy(plan)


@pytest.mark.gpu
def test_gpu_errors_are_reported_with_messages():
    """capi/tests/c_api.rs:433-507 with a GPU plan."""
    _gpu()
    assert makeplan(1, [8], eps=1e-20)[0] == 2
    code, plan = makeplan(1, [8])
    assert code == 0, last_error()
    try:
        f = np.zeros(16)
        c = np.zeros(2)
        assert lib.wgpu_nufft_execute(plan, ptr(c), ptr(f)) == 1 and "set the points" in last_error()
        far = np.array([10.0])
        assert lib.wgpu_nufft_setpts(plan, 1, ptr(far), None, None, 0, None, None, None) == 1
        assert "3*pi" in last_error()
        nan = np.array([np.nan])
        assert lib.wgpu_nufft_setpts(plan, 1, ptr(nan), None, None, 0, None, None, None) == 1
        assert lib.wgpu_nufft_setpts(plan, 1, None, None, None, 0, None, None, None) == 1
        assert lib.wgpu_nufftf_execute(plan, None, None) == 1 and "array type" in last_error()
        # A failed setpts leaves the plan without points.
        assert lib.wgpu_nufft_execute(plan, ptr(c), ptr(f)) == 1 and "set the points" in last_error()
        ok = np.array([0.5])
        assert lib.wgpu_nufft_setpts(plan, 1, ptr(ok), None, None, 0, None, None, None) == 0
        bad = np.array([np.inf, 0.0])
        assert lib.wgpu_nufft_execute(plan, ptr(bad), ptr(f)) == 1 and "finite" in last_error()
        good = np.array([1.0, 0.0])
        assert lib.wgpu_nufft_execute(plan, ptr(good), ptr(f)) == 0, last_error()
        ref = native.direct_type1(ok[:, None], np.array([[1.0 + 0j]]), [8], 1)[0]
        assert rel_l2(complex_of(f), ref) < 1e-5
        # More than eight dimensions are an argument error.
        assert makeplan(1, [2] * 9)[0] == 1 and "between 1 and 8" in last_error()
    finally:
        lib.wgpu_nufft_destroy(plan)


@pytest.mark.gpu
def test_gpu_type3_plans_take_bounds_from_their_points():
    """capi/src/plan.rs:353-397: bounds from the points, rebuilt only when a
    later set leaves them; batches of ntrans strengths."""
    _gpu()
    rng = np.random.default_rng(33)
    ntrans = 2
    plan = ctypes.c_void_p()
    assert lib.wgpu_nufft_makeplan(3, 2, None, 1, ntrans, 1e-9, ctypes.byref(plan), None) == 0, last_error()
    try:
        for scale in (1.0, 0.5, 2.0):
            m, n = 400, 300
            src = rng.uniform(-scale, scale, (m, 2))
            tgt = rng.uniform(-30 * scale, 30 * scale, (n, 2))
            srcc, tgtc = np.ascontiguousarray(src), np.ascontiguousarray(tgt)
            assert lib.wgpu_nufft_setpts_nd(plan, m, ptr(srcc), n, ptr(tgtc)) == 0, last_error()
            c = rng.standard_normal((ntrans, m)) + 1j * rng.standard_normal((ntrans, m))
            out = np.zeros(2 * n * ntrans)
            assert lib.wgpu_nufft_execute(plan, ptr(interleaved(c)), ptr(out)) == 0, last_error()
            ref = native.direct_type3(src, c, tgt, 1)
            assert rel_l2(complex_of(out).reshape(ntrans, n), ref) < 1e-7, scale
        # Empty sets.
        assert lib.wgpu_nufft_setpts_nd(plan, 0, None, 0, None) == 0, last_error()
        assert lib.wgpu_nufft_execute(plan, None, None) == 0, last_error()
    finally:
        lib.wgpu_nufft_destroy(plan)


@pytest.mark.gpu
def test_gpu_empty_point_sets():
    _gpu()
    f = np.full(2 * 12, 7.0)
    assert lib.wgpu_nufft1d1(0, None, None, 1, 1e-6, 12, ptr(f), None) == 0, last_error()
    assert np.all(f == 0.0)
    fm = np.ones(2 * 12)
    assert lib.wgpu_nufft1d2(0, None, None, 1, 1e-6, 12, ptr(fm), None) == 0, last_error()


@pytest.mark.gpu
def test_gpu_adapters_are_listed_and_selected():
    """capi/tests/c_api.rs:530-665 on this box's CUDA devices."""
    _gpu()
    count = ctypes.c_int32()
    assert lib.wgpu_nufft_list_adapters(None, 0, ctypes.byref(count)) == 0
    assert count.value >= 1
    adapters = (_native.WgpuAdapter * count.value)()
    assert lib.wgpu_nufft_list_adapters(adapters, count.value, ctypes.byref(count)) == 0
    assert [a.is_default for a in adapters].count(1) == 1 and adapters[0].is_default == 1
    for a in adapters:
        assert a.name and a.backend == b"CUDA" and a.device_type == b"DiscreteGpu"
    first = adapters[0]
    one = (_native.WgpuAdapter * 1)()
    assert lib.wgpu_nufft_list_adapters(one, 1, ctypes.byref(count)) == 0
    assert bytes(one[0]) == bytes(first) and count.value == len(adapters)

    lib.wgpu_nufft_shutdown()
    x = np.linspace(-3, 3, 40)
    c = np.ones(80)
    f = np.zeros(32)

    def type1_with(o):
        return lib.wgpu_nufft1d1(40, ptr(x), ptr(c), 1, 1e-6, 16, ptr(f), ctypes.byref(o))

    assert type1_with(opts(GPU)) == 0, last_error()
    assert lib.wgpu_nufft_gpu_name().decode() == first.name.decode() + " (CUDA)"
    lib.wgpu_nufft_shutdown()
    same_name = sum(1 for a in adapters if a.name == first.name)
    by_name = opts(name=first.name.upper(), index=1 if same_name > 1 else 0)
    assert type1_with(by_name) == 0, last_error()
    assert type1_with(opts(index=1)) == 0, last_error()
    if first.pci_bus_id:
        assert type1_with(opts(pci=first.pci_bus_id)) == 0, last_error()
    assert type1_with(opts(name=b"No Such Adapter 7f3a")) == 3
    assert 'no GPU adapter matches name "No Such Adapter 7f3a"' in last_error()
    assert type1_with(opts(index=10_000)) == 3 and "index 10000" in last_error()
    if len(adapters) > 1:
        assert type1_with(opts(index=2)) == 1 and "wgpu_nufft_shutdown" in last_error()
    lib.wgpu_nufft_shutdown()


@pytest.mark.gpu
def test_gpu_four_dimensional_plans_through_setpts_nd():
    """Plans of more than three dimensions take point-major coordinates
    through setpts_nd and match FP64 direct sums (type 1 and type 2)."""
    rng = np.random.default_rng(44)
    n_modes = [4, 3, 5, 2]
    m = 300
    pts = rng.uniform(-np.pi, np.pi, (m, 4))
    for kind in (1, 2):
        code, plan = makeplan(kind, n_modes, eps=1e-6)
        assert code == 0, last_error()
        try:
            assert lib.wgpu_nufft_setpts_nd(plan, m, ptr(pts), 0, None) == 0, last_error()
            if kind == 1:
                c = rng.standard_normal(2 * m)
                f = np.zeros(2 * int(np.prod(n_modes)))
                assert lib.wgpu_nufft_execute(plan, ptr(c), ptr(f)) == 0, last_error()
                ref = native.direct_type1(pts, complex_of(c)[None, :], n_modes, 1)[0]
                assert rel_l2(complex_of(f), ref) < 1e-5
            else:
                f = rng.standard_normal(2 * int(np.prod(n_modes)))
                c = np.zeros(2 * m)
                # execute(plan, c, f): values at the points, then modes.
                assert lib.wgpu_nufft_execute(plan, ptr(c), ptr(f)) == 0, last_error()
                ref = native.direct_type2(pts, complex_of(f)[None, :], n_modes, 1)[0]
                assert rel_l2(complex_of(c), ref) < 1e-5
        finally:
            lib.wgpu_nufft_destroy(plan)
