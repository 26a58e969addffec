"""ES window mathematics restated from src/kernel.rs (oracle; test infrastructure)."""

from __future__ import annotations

import math

import numpy as np

MIN_WIDTH = 2
MAX_WIDTH = 16
MAX_HORNER_COEFFICIENTS = 19
MAX_FINE_GRID_LENGTH = 2**32 - 1


class OracleError(ValueError):
    def __init__(self, kind: str, message: str = ""):
        self.kind = kind
        super().__init__(f"{kind}: {message}")


def es_parameters(eps: float, sigma: float = 2.0) -> tuple[int, float]:
    """(width, beta) of EsKernel::for_tolerance (src/kernel.rs:21-57)."""
    if not math.isfinite(eps) or not (0.0 < eps < 1.0):
        raise OracleError("InvalidTolerance")
    if not math.isfinite(sigma) or sigma <= 1.0:
        raise OracleError("InvalidSigma")
    if sigma == 2.0:
        width_float = math.ceil(math.log10(10.0 / eps))
    else:
        width_float = math.log(1.0 / eps) / (math.pi * math.sqrt(1.0 - 1.0 / sigma))
    width = max(int(math.ceil(width_float)), MIN_WIDTH)
    if width > MAX_WIDTH:
        raise OracleError("KernelWidthUnsupported")
    if sigma == 2.0:
        beta = {2: 2.20, 3: 2.26, 4: 2.38}.get(width, 2.30) * width
    else:
        beta = 0.97 * math.pi * width * (1.0 - 1.0 / (2.0 * sigma))
    return width, beta


def es_evaluate(width: int, beta: float, distance):
    """EsKernel::evaluate (src/kernel.rs:81-89), vectorised."""
    d = np.abs(np.asarray(distance, dtype=np.float64))
    half = 0.5 * width
    with np.errstate(invalid="ignore"):
        inside = np.isfinite(d) & (d < half)
        scaled = np.where(inside, 2.0 * d / width, 0.0)
        value = np.exp(beta * (np.sqrt(1.0 - scaled * scaled) - 1.0))
    return np.where(inside, value, 0.0)


def _chebyshev_fit(function, count: int) -> list[float]:
    """polynomial_fit_chebyshev (src/kernel.rs:240-271): highest degree first."""
    nodes = [math.cos(((2 * i + 1) * math.pi) / (2 * count)) for i in range(count)]
    divided = [float(function(x)) for x in nodes]
    for order in range(1, count):
        for index in range(count - 1, order - 1, -1):
            divided[index] = (divided[index] - divided[index - 1]) / (nodes[index] - nodes[index - order])
    coefficients = [0.0] * count
    basis = [1.0]
    coefficients[0] = divided[0]
    for order in range(1, count):
        node = nodes[order - 1]
        nxt = [0.0] * (len(basis) + 1)
        for power, value in enumerate(basis):
            nxt[power] -= node * value
            nxt[power + 1] += value
        basis = nxt
        for power, value in enumerate(basis):
            coefficients[power] += divided[order] * value
    return coefficients[::-1]


def horner_table(width: int, beta: float, eps: float) -> tuple[int, np.ndarray]:
    """EsKernel::horner_table (src/kernel.rs:93-130): (rows, coefficient-major table)."""
    fitted = min(width + 3, MAX_HORNER_COEFFICIENTS)
    table = np.zeros((fitted, width))
    for panel in range(width):
        shift = float(2 * panel + 1) - width
        fit = _chebyshev_fit(lambda t: float(es_evaluate(width, beta, (t + shift) * 0.5)), fitted)
        table[:, panel] = fit
    minimum = max(4, max(width - 4, 0))
    threshold = 0.05 * eps
    leading = 0
    while fitted - leading > minimum and np.all(np.abs(table[leading]) < threshold):
        leading += 1
    return fitted - leading, table[leading:].copy()


def horner_evaluate(width: int, table: np.ndarray, distance: float) -> float:
    """EsHornerTable::evaluate (src/kernel.rs:221-236)."""
    half = 0.5 * width
    if not math.isfinite(distance) or abs(distance) >= half:
        return 0.0
    panel = min(max(int(math.ceil(distance + half)) - 1, 0), width - 1)
    local = 2.0 * (distance - panel) + (width - 1)
    value = 0.0
    for row in table[:, panel]:
        value = value * local + row
    return value


def _legendre_pair(order: int, x: float) -> tuple[float, float]:
    previous = 1.0
    if order == 0:
        return previous, 0.0
    current = x
    for degree in range(2, order + 1):
        nxt = ((2 * degree - 1) * x * current - (degree - 1) * previous) / degree
        previous, current = current, nxt
    return current, previous


def gauss_legendre(order: int) -> tuple[np.ndarray, np.ndarray]:
    """gauss_legendre (src/kernel.rs:367-392)."""
    nodes = np.zeros(order)
    weights = np.zeros(order)
    eps64 = np.finfo(np.float64).eps
    for index in range((order + 1) // 2):
        root = math.cos(math.pi * (index + 0.75) / (order + 0.5))
        while True:
            p, q = _legendre_pair(order, root)
            derivative = order * (root * p - q) / (root * root - 1.0)
            nxt = root - p / derivative
            done = abs(nxt - root) <= 4.0 * eps64
            root = nxt
            if done:
                break
        p, q = _legendre_pair(order, root)
        derivative = order * (root * p - q) / (root * root - 1.0)
        weight = 2.0 / ((1.0 - root * root) * derivative * derivative)
        nodes[index], nodes[order - 1 - index] = -root, root
        weights[index] = weights[order - 1 - index] = weight
    return nodes, weights


def centered_fourier_coefficients(width: int, beta: float, fine_length: int, table=None) -> np.ndarray:
    """phi_hat[k], k = 0..n/2, with (-1)^k (src/kernel.rs:134-198)."""
    if fine_length % 2:
        raise OracleError("FineGridMustBeEven")
    half = 0.5 * width
    q = int(math.floor(2.0 + 3.0 * half))
    nodes, weights = gauss_legendre(2 * q)
    qn = half * nodes[:q]
    if table is None:
        kv = es_evaluate(width, beta, qn)
    else:
        kv = np.array([horner_evaluate(width, table, x) for x in qn])
    wk = half * weights[:q] * kv
    modes = np.arange(fine_length // 2 + 1)
    freq = 2.0 * math.pi * modes / fine_length
    values = np.array([sum(2.0 * wk[i] * math.cos(f * qn[i]) for i in range(q)) for f in freq])
    values[1::2] *= -1.0
    return values


def fft_length_supported(length: int) -> bool:
    if length <= 0:
        return False
    for radix in (2, 3, 5, 7, 11):
        while length % radix == 0:
            length //= radix
    return length == 1


def select_fine_grid_size(n_modes: int, sigma: float, width: int) -> int:
    """select_fine_grid_size (src/kernel.rs:278-333) over radices 2, 3, 5, 7, 11."""
    if n_modes == 0:
        raise OracleError("ZeroMode")
    if not (MIN_WIDTH <= width <= MAX_WIDTH):
        raise OracleError("InvalidKernelWidth")
    if not math.isfinite(sigma) or sigma <= 1.0:
        raise OracleError("InvalidSigma")
    scaled = 2 * n_modes if sigma == 2.0 else int(math.ceil(sigma * n_modes))
    minimum = max(scaled, 2 * width)
    candidate = minimum if minimum % 2 == 0 else minimum + 1
    while candidate <= MAX_FINE_GRID_LENGTH:
        if fft_length_supported(candidate):
            return candidate
        candidate += 2
    raise OracleError("FineGridTooLarge", str(minimum))


def mode_for_storage_index(order: int, index, length: int):
    """mode_for_storage_index (src/direct.rs:120-131); order 0 centered, 1 FFT."""
    index = np.asarray(index)
    if order == 0:
        return index - length // 2
    return np.where(index < (length + 1) // 2, index, index - length)


def mode_amplitudes(n_modes, order: int, coefficients) -> np.ndarray:
    """prod_a 1/phi_hat_a(|k_a|) over the mode box, axis 0 fastest, in f64
    (mode_amplitudes_nd, src/gpu_nd.rs:910-951)."""
    amplitude = np.ones(1)
    # Built from the last axis outward so that axis 0 is fastest; each mode's
    # divisions still run in axis order 0, 1, ... as in the reference.
    grids = np.meshgrid(*[np.arange(n) for n in n_modes], indexing="ij")
    amplitude = np.ones(grids[0].shape)
    for axis, n in enumerate(n_modes):
        modes = mode_for_storage_index(order, grids[axis], n)
        amplitude = amplitude / np.asarray(coefficients[axis])[np.abs(modes)]
    return amplitude.transpose().reshape(-1)
