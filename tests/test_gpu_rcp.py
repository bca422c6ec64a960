"""The factor and per-step kernels' FP64 reciprocal (rcp_nr: the hardware
approximation refined by two Newton-Raphson steps, inline instead of CUDA's
division routine) against the exact reciprocal: at most 1 ulp over the
normal range, exact on powers of two, and the sign kept."""
import numpy as np
import pytest

from conftest import load_package

load_package()
from croma_fp_b200 import native  # noqa: E402

pytestmark = pytest.mark.gpu


def ulp_err(y, x):
    ref = 1.0 / x
    return np.abs(y - ref) / np.spacing(np.abs(ref))


def test_reciprocal_within_one_ulp():
    rng = np.random.default_rng(7)
    n = 1 << 20
    # mantissas uniform in [1, 2), exponents over the range where 1/x is normal too
    x = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-1000, 1000, n)) * rng.choice([-1.0, 1.0], n)
    y = native.rcp_check(x)
    assert np.all(np.sign(y) == np.sign(x))
    assert float(np.max(ulp_err(y, x))) <= 1.0


def test_reciprocal_on_the_operand_ranges_of_the_kernels():
    """Pivot denominators (1 + O(dt) terms) and face-weight denominators
    (1 - exp(-|w|) for |w| >= 0.1, exp(w/2) times the series for |w| < 0.1)."""
    rng = np.random.default_rng(8)
    w = np.concatenate([rng.uniform(0.1, 700.0, 1 << 16), rng.uniform(-0.1, 0.1, 1 << 16)])
    dser = 1.0 + w * w / 24.0 + w ** 4 / 1920.0
    den = np.where(np.abs(w) < 0.1, np.exp(0.5 * w) * dser, 1.0 - np.exp(-np.abs(w)))
    piv = 1.0 + rng.uniform(0.0, 1e6, 1 << 16) * rng.uniform(0.0, 1.0, 1 << 16)
    for x in (den, piv):
        assert float(np.max(ulp_err(native.rcp_check(x), x))) <= 1.0


def test_reciprocal_exact_on_powers_of_two():
    x = np.exp2(np.arange(-1000, 1001, dtype=np.float64))
    assert np.array_equal(native.rcp_check(x), 1.0 / x)
