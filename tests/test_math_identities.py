"""Identities the device code relies on, checked against the host C library the
reference links (no GPU needed).

The viscosity update evaluates the reference's pow(v, 0.5) (strain-rate and stress
invariants, markmart.c:47-48; the Peierls iteration of viscalc, markmart.c:1923)
as sqrt(v), with pow's results for -0 (+0) and -inf (+inf).  glibc's pow is not
correctly rounded, so for a small fraction of doubles the two differ by one unit
in the last place; never by more, and never in the special values."""
import ctypes as C
import ctypes.util

import numpy as np

libm = C.CDLL(ctypes.util.find_library("m"))
libm.pow.restype = C.c_double
libm.pow.argtypes = [C.c_double, C.c_double]
libm.sqrt.restype = C.c_double
libm.sqrt.argtypes = [C.c_double]


def pow_half(v: float) -> float:
    """The device's evaluation (i2g_dev.cuh: pow_half)."""
    return float("inf") if v == float("-inf") else libm.sqrt(v) + 0.0


def ulps(a: float, b: float) -> int:
    if np.isnan(a) and np.isnan(b):
        return 0
    ia, ib = np.float64(a).view(np.int64), np.float64(b).view(np.int64)
    return abs(int(ia) - int(ib))


def test_sqrt_within_one_ulp_of_pow_half():
    rng = np.random.default_rng(20261203)
    values = np.concatenate([
        rng.random(20000) * 10.0 ** rng.integers(-300, 300, 20000),   # positive normals
        np.frombuffer(rng.integers(1, 2 ** 52, 2000, dtype=np.uint64).tobytes(), dtype=np.float64),  # subnormals
        -rng.random(200),                                            # negatives: NaN from both
        np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 1.7976931348623157e308, 1.0, 4.0]),
    ])
    diff = np.array([ulps(pow_half(float(v)), libm.pow(float(v), 0.5)) for v in values])
    assert diff.max() <= 1
    assert (diff > 0).mean() < 0.01
    for v in (0.0, -0.0, np.inf, -np.inf, np.nan, -1.0, 1.0, 4.0, 5e-324):
        assert ulps(pow_half(v), libm.pow(v, 0.5)) == 0, v
        assert np.signbit(pow_half(v)) == np.signbit(libm.pow(v, 0.5)) or np.isnan(v) or v < 0, v
