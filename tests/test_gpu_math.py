"""The factor and per-step kernels' own FP64 math, against exact values:
the reciprocal rcp_nr (the hardware approximation refined by two
Newton-Raphson steps, inline instead of CUDA's division routine) -- at most
1 ulp over the normal range, exact on powers of two, the sign kept -- and the
table-driven exponential exp_tab (Tang's method) -- at most 1 ulp against a
multiprecision exp over the factor kernels' argument range and beyond, exact
at 0, and 0 far below the subnormal range."""
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


def _exp_ulp(y, x):
    mp = pytest.importorskip("mpmath")
    mp.mp.prec = 120
    worst = 0.0
    for xi, yi in zip(x, y):
        ref = mp.exp(mp.mpf(float(xi)))
        if ref < mp.mpf(2) ** -1022:
            continue
        ulp = mp.mpf(2) ** (mp.floor(mp.log(ref, 2)) - 52)
        worst = max(worst, float(abs(mp.mpf(float(yi)) - ref) / ulp))
    return worst


def test_exponential_within_one_ulp():
    rng = np.random.default_rng(9)
    # face weights: exp(w/2) for |w| < 0.1 and exp(-|w|) for |w| >= 0.1;
    # Coulomb: exp(-x) for x in [0, 40]; plus the rest of the range
    x = np.concatenate([rng.uniform(-0.05, 0.05, 4000), rng.uniform(-40.0, -0.1, 4000),
                        rng.uniform(-708.0, -40.0, 2000), rng.uniform(0.0, 700.0, 2000)])
    y = native.exp_check(x)
    assert _exp_ulp(y, x) <= 1.0


def test_exponential_edges():
    x = np.array([0.0, -0.0, -746.0, -800.0, -1e300, 1e-300, -1e-300, np.nan])
    y = native.exp_check(x)
    assert y[0] == 1.0 and y[1] == 1.0 and y[5] == 1.0 and y[6] == 1.0
    assert y[2] == 0.0 and y[3] == 0.0 and y[4] == 0.0 and np.isnan(y[7])
    # results in the subnormal range are formed, not flushed
    xs = np.array([-710.0, -730.0, -744.0])
    ys = native.exp_check(xs)
    assert np.all(ys > 0.0) and np.all(np.abs(ys - np.exp(xs)) <= 2.0 ** -1074 * 2)
