"""The NumPy plans (wgpunufft_b200.numpy_api) against the reference's Python
binding tests (python/tests/test_bindings.py): direct sums, NumPy axis
order, batches, concurrent calls on one plan, type 3, empty transforms,
validation messages, the error type's pickle round trip, a clean shutdown of
a fresh process and plans destroyed on another thread."""

from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import native

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

from wgpunufft_b200 import numpy_api as wn  # noqa: E402


@pytest.fixture(scope="module")
def context():
    return wn.Context()


def _direct1(points, strengths, n_modes, isign, order):
    """Oracle type-1 sums in the NumPy layout of n_modes."""
    pts = np.asarray(points, np.float64).reshape(-1, len(n_modes))
    c = np.atleast_2d(np.asarray(strengths, np.complex128))
    core = native.direct_type1(pts, c, n_modes, isign, order)
    d = len(n_modes)
    out = core.reshape((c.shape[0],) + tuple(reversed(n_modes))).transpose((0,) + tuple(range(d, 0, -1)))
    return out[0] if np.ndim(strengths) == 1 else out


def _direct2(points, coefficients, n_modes, isign, order):
    pts = np.asarray(points, np.float64).reshape(-1, len(n_modes))
    d = len(n_modes)
    f = np.asarray(coefficients, np.complex128).reshape((-1,) + tuple(n_modes))
    core = np.ascontiguousarray(f.transpose((0,) + tuple(range(d, 0, -1)))).reshape(f.shape[0], -1)
    out = native.direct_type2(pts, core, n_modes, isign, order)
    return out[0] if np.ndim(coefficients) == d else out


def _close(actual, expected):
    scale = max(1.0, float(np.max(np.abs(expected), initial=0.0)))
    np.testing.assert_allclose(actual, expected, rtol=5e-3, atol=5e-3 * scale)


@pytest.mark.parametrize("isign", [-1, 1])
@pytest.mark.parametrize("mode_order", ["centered", "fft"])
def test_type1_and_type2_1d_match_direct(context, isign, mode_order):
    points = np.array([-2.1, -0.4, 0.0, 0.7, 2.4], dtype=np.float32)
    strengths = np.array([1.0 + 0.2j, -0.4 + 0.7j, 0.3 - 0.1j, 1.2 + 0.5j, -0.2 - 0.8j], dtype=np.complex64)
    coefficients = np.array([0.1 + 0.3j, -0.2 + 0.4j, 0.8 - 0.1j, 0.5 + 0.2j, -0.7 + 0.6j, 0.2 - 0.5j, 0.9],
                            dtype=np.complex64)
    order = 0 if mode_order == "centered" else 1
    type1 = wn.Type1Plan(context, (7,), eps=1e-4, isign=isign, mode_order=mode_order)
    actual1 = type1.execute(points, strengths)
    assert actual1.dtype == np.complex64 and actual1.shape == (7,)
    _close(actual1, _direct1(points, strengths, (7,), isign, order))
    type2 = wn.Type2Plan(context, (7,), eps=1e-4, isign=isign, mode_order=mode_order)
    actual2 = type2.execute(points, coefficients)
    assert actual2.dtype == np.complex64 and actual2.shape == (5,)
    _close(actual2, _direct2(points, coefficients, (7,), isign, order))


def test_non_square_2d_numpy_axis_order(context):
    points = np.array([[-1.2, 0.4], [0.1, -0.7], [1.0, 1.3], [2.2, -1.8]], dtype=np.float32)
    strengths = np.array([1.0 + 0.1j, -0.3 + 0.8j, 0.5 - 0.2j, -0.7 - 0.4j], dtype=np.complex64)
    modes = wn.Type1Plan(context, (3, 5), eps=1e-4).execute(points, strengths)
    assert modes.shape == (3, 5)
    _close(modes, _direct1(points, strengths, (3, 5), 1, 0))
    coefficients = (np.arange(15, dtype=np.float32).reshape(3, 5) / 10
                    + 1j * np.flip(np.arange(15, dtype=np.float32).reshape(3, 5)) / 20).astype(np.complex64)
    values = wn.Type2Plan(context, (3, 5), eps=1e-4).execute(points, coefficients)
    _close(values, _direct2(points, coefficients, (3, 5), 1, 0))


def test_3d_numpy_axis_order(context):
    rng = np.random.default_rng(3)
    n_modes = (3, 4, 5)
    points = rng.uniform(-np.pi, np.pi, (9, 3)).astype(np.float32)
    strengths = (rng.standard_normal(9) + 1j * rng.standard_normal(9)).astype(np.complex64)
    modes = wn.Type1Plan(context, n_modes, eps=1e-4, isign=-1).execute(points, strengths)
    assert modes.shape == n_modes
    _close(modes, _direct1(points, strengths, n_modes, -1, 0))
    coefficients = (rng.standard_normal(n_modes) + 1j * rng.standard_normal(n_modes)).astype(np.complex64)
    values = wn.Type2Plan(context, n_modes, eps=1e-4, isign=-1).execute(points, coefficients)
    assert values.shape == (9,)
    _close(values, _direct2(points, coefficients, n_modes, -1, 0))


def test_batched_reuse_and_explicit_batch_axis(context):
    points = np.array([-1.3, -0.2, 0.5, 1.7], dtype=np.float32)
    strengths = np.array([[1.0, 0.2 + 0.4j, -0.3 + 0.1j, 0.7 - 0.5j],
                          [-0.2 + 0.8j, 0.9 + 0.1j, 0.1 - 0.6j, 0.4 + 0.3j],
                          [0.3 - 0.2j, -0.5 + 0.7j, 1.1, -0.1 - 0.4j]], dtype=np.complex64)
    plan = wn.Type1Plan(context, (6,), eps=1e-4, batch=3)
    batched = plan.execute(points, strengths)
    assert batched.shape == (3, 6)
    for t in range(3):
        _close(batched[t], _direct1(points, strengths[t], (6,), 1, 0))
    single = plan.execute(points, strengths[0])
    repeated = plan.execute(points, strengths[0:1])
    assert single.shape == (6,) and repeated.shape == (1, 6)
    np.testing.assert_array_equal(repeated[0], single)


def test_same_plan_serializes_concurrent_calls(context):
    plan = wn.Type1Plan(context, (8,), eps=1e-4)
    large_points = np.linspace(-2.5, 2.5, 32, dtype=np.float32)
    large = (np.linspace(-0.7, 0.9, 32) + 1j * np.linspace(0.6, -0.4, 32)).astype(np.complex64)
    small_points = np.array([-1.1, 0.2, 1.4], dtype=np.float32)
    small = np.array([0.3 + 0.8j, -0.5 + 0.1j, 0.9 - 0.4j], dtype=np.complex64)
    with ThreadPoolExecutor(max_workers=2) as pool:
        f1 = pool.submit(plan.execute, large_points, large)
        f2 = pool.submit(plan.execute, small_points, small)
        got_large, got_small = f1.result(), f2.result()
    _close(got_large, _direct1(large_points, large, (8,), 1, 0))
    _close(got_small, _direct1(small_points, small, (8,), 1, 0))
    np.testing.assert_array_equal(got_small, plan.execute(small_points, small))


def test_type3_batched_matches_direct(context):
    source = np.array([[-0.8, 0.3], [0.2, -0.5], [0.9, 0.7]], dtype=np.float32)
    target = np.array([[-1.2, 0.1], [0.4, -0.9], [1.1, 0.8], [1.7, -1.4]], dtype=np.float32)
    strengths = np.array([[1.0 + 0.2j, -0.3 + 0.7j, 0.4 - 0.5j],
                          [-0.2 + 0.1j, 0.8 - 0.4j, 0.6 + 0.3j]], dtype=np.complex64)
    plan = wn.Type3Plan(context, [[-1.0, 1.0], [-1.0, 1.0]], [[-2.0, 2.0], [-2.0, 2.0]], eps=1e-4,
                        isign=-1, batch=2)
    actual = plan.execute(source, strengths, target)
    assert actual.shape == (2, 4)
    ref = native.direct_type3(source.astype(np.float64), strengths.astype(np.complex128),
                              target.astype(np.float64), -1)
    for t in range(2):
        _close(actual[t], ref[t])
    assert plan.outer_grid_shape == [int(n) for n in plan.outer_grid_shape]


def test_empty_transforms_have_mathematical_shapes(context):
    empty_points = np.empty(0, dtype=np.float32)
    empty_values = np.empty(0, dtype=np.complex64)
    type1 = wn.Type1Plan(context, (5,), eps=1e-4)
    np.testing.assert_array_equal(type1.execute(empty_points, empty_values), np.zeros(5, dtype=np.complex64))
    type2 = wn.Type2Plan(context, (5,), eps=1e-4)
    assert type2.execute(empty_points, np.ones(5, dtype=np.complex64)).shape == (0,)
    bounds = np.array([[-1.0, 1.0]])
    type3 = wn.Type3Plan(context, bounds, bounds, eps=1e-4)
    target = np.array([-0.5, 0.25], dtype=np.float32)
    np.testing.assert_array_equal(type3.execute(empty_points, empty_values, target),
                                  np.zeros(2, dtype=np.complex64))


def test_validation_errors_are_clear(context):
    plan = wn.Type1Plan(context, (5,), eps=1e-4)
    values = np.ones(3, dtype=np.complex64)
    with pytest.raises(TypeError):
        plan.execute(np.zeros(3, dtype=np.float64), values)
    with pytest.raises(ValueError, match="C-contiguous"):
        plan.execute(np.arange(6, dtype=np.float32)[::2], values)
    with pytest.raises(ValueError, match="non-finite"):
        plan.execute(np.array([0.0, np.nan, 1.0], dtype=np.float32), values)
    with pytest.raises(ValueError, match=r"outside \[-3\*pi, 3\*pi\]"):
        plan.execute(np.array([0.0, 10.0, 1.0], dtype=np.float32), values)
    with pytest.raises(ValueError, match="plan capacity"):
        plan.execute(np.zeros(3, dtype=np.float32), np.ones((2, 3), dtype=np.complex64))
    with pytest.raises(ValueError, match="isign"):
        wn.Type1Plan(context, (5,), isign=2)
    with pytest.raises(ValueError, match="mode_order"):
        wn.Type1Plan(context, (5,), mode_order="natural")
    bounds = np.array([[-1.0, 1.0]])
    type3 = wn.Type3Plan(context, bounds, bounds, eps=1e-4)
    with pytest.raises(ValueError, match="outside"):
        type3.execute(np.array([1.1], dtype=np.float32), np.ones(1, dtype=np.complex64),
                      np.array([0.0], dtype=np.float32))
    with pytest.raises(ValueError, match="endpoint"):
        wn.Type3Plan(context, [[1.0, -1.0]], bounds)


def test_context_describes_the_device(context):
    assert context.backend == "CUDA"
    assert context.adapter_name
    assert context.device_type == "DiscreteGpu"
    with pytest.raises(wn.WgpuNufftError):
        wn.Context(force_fallback=True)


ROOT = __import__("pathlib").Path(__file__).resolve().parents[1]


def _run_script(script: str):
    import subprocess
    import sys

    return subprocess.run([sys.executable, "-c", script], cwd=str(ROOT), check=False, capture_output=True,
                          text=True, timeout=300)


def test_error_pickles_and_the_interface_is_documented():
    """The reference's metadata test (test_bindings.py:18-25): the error type
    survives a pickle round trip with its message, and the plans document
    themselves."""
    import pickle

    error = pickle.loads(pickle.dumps(wn.WgpuNufftError("test error")))
    assert isinstance(error, wn.WgpuNufftError)
    assert str(error) == "test error"
    assert wn.Context.__doc__
    assert wn.Type1Plan.execute.__doc__
    assert wn.Type2Plan.execute.__doc__


def test_gpu_resources_shut_down_cleanly_in_a_fresh_process():
    """A process that makes a context and a plan, executes and exits without
    releasing them ends with status 0 (test_bindings.py:28-46)."""
    completed = _run_script("""
import numpy as np
from wgpunufft_b200 import numpy_api as wn

context = wn.Context()
plan = wn.Type1Plan(context, (8,), eps=1e-4)
points = np.array([-0.5, 0.25], dtype=np.float32)
strengths = np.array([1.0 + 0.2j, -0.3 + 0.4j], dtype=np.complex64)
plan.execute(points, strengths)
""")
    assert completed.returncode == 0, completed.stderr


def test_gpu_plans_can_be_destroyed_on_another_thread():
    """Plans made on the main thread and released on a worker thread (after
    their context is gone) leave the process healthy (test_bindings.py:49-90)."""
    completed = _run_script("""
import gc
import queue
import threading

from wgpunufft_b200 import numpy_api as wn

objects = queue.Queue()
stop = object()

def worker():
    while True:
        obj = objects.get()
        if obj is stop:
            objects.task_done()
            return
        del obj
        gc.collect()
        objects.task_done()

thread = threading.Thread(target=worker)
thread.start()
for _ in range(8):
    context = wn.Context()
    plan = wn.Type1Plan(context, (8,), eps=1e-4)
    del context
    objects.put(plan)
    del plan
    objects.join()
objects.put(stop)
objects.join()
thread.join()
""")
    assert completed.returncode == 0, completed.stderr
