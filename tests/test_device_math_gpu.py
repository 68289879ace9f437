"""Device arithmetic that must equal the host's bit for bit (see vh_math.cuh
and div_rcp in vh_physics.cuh), checked on the GPU against the host libm and
IEEE division on millions of inputs."""
import ctypes as C

import numpy as np
import pytest

import vh

pytestmark = pytest.mark.gpu
libm = C.CDLL("libm.so.6")
libm.tanh.restype = C.c_double
libm.tanh.argtypes = [C.c_double]
libm.powf.restype = C.c_float
libm.powf.argtypes = [C.c_float, C.c_float]


def test_tanh_matches_host_libm():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(0, 1e-7, 50000), rng.uniform(0, 1, 400000), rng.uniform(0, 25, 400000),
                        rng.exponential(0.05, 150000), -rng.uniform(0, 3, 100000), [0.0, 1e-300, 22.0, 0.5493, 1.0]])
    dev = vh.device_math(0, x)
    host = np.array([libm.tanh(v) for v in x])
    assert np.array_equal(dev.view(np.uint64), host.view(np.uint64)), int((dev != host).sum())


def test_shared_reciprocal_division_is_ieee():
    rng = np.random.default_rng(2)
    n = 4_000_000
    a = np.ldexp(rng.uniform(1, 2, n), rng.integers(-300, 300, n)) * rng.choice([-1, 1], n)
    b = np.ldexp(rng.uniform(1, 2, n), rng.integers(-300, 300, n)) * rng.choice([-1, 1], n)
    b[::7] = 3.0
    b[::11] = 0.15
    a[::13] = 0.0
    q_rcp = vh.device_math(1, a, b)
    q_ieee = vh.device_math(2, a, b)
    assert np.array_equal(q_rcp.view(np.uint64), q_ieee.view(np.uint64))
    assert np.array_equal(q_ieee.view(np.uint64), (a / b).view(np.uint64))


def test_shared_reciprocal_division_edge_operands():
    """signed zeros (the zero-numerator shortcut), infinities, NaN,
    subnormals, operands at the fast path's thresholds (2^-960, 2^1000)
    and every exponent: equal to IEEE a / b bit for bit (NaN as NaN)"""
    rng = np.random.default_rng(4)
    special = np.array([0.0, -0.0, 1.0, -1.0, 3.0, 0.15, np.inf, -np.inf, np.nan, 5e-324, -5e-324, 1e-310,
                        2.2250738585072014e-308, 1.7976931348623157e308, -1.7976931348623157e308,
                        2.0 ** -960, -(2.0 ** -960), 2.0 ** -961, 2.0 ** 1000, 2.0 ** 999, 2.0 ** 1001, 2.0 ** 960,
                        2.0 ** 961])
    sa, sb = np.meshgrid(special, special)
    n = 2_000_000
    bits = rng.integers(0, 2 ** 63, n, dtype=np.uint64) | (rng.integers(0, 2, n, dtype=np.uint64) << np.uint64(63))
    a = np.concatenate([sa.ravel(), bits.view(np.float64), np.zeros(1000), -np.zeros(1000)])
    bits = rng.integers(0, 2 ** 63, a.size, dtype=np.uint64)
    b = bits.view(np.float64).copy()
    b[:sb.size] = sb.ravel()
    b[-2000:] = rng.uniform(0.5, 4.0, 2000) * rng.choice([-1, 1], 2000)
    q_rcp = vh.device_math(1, a, b)
    with np.errstate(all="ignore"):
        q_host = a / b
    both_nan = np.isnan(q_rcp) & np.isnan(q_host)
    same = q_rcp.view(np.uint64) == q_host.view(np.uint64)
    assert np.all(same | both_nan), int((~(same | both_nan)).sum())
    zero = np.isfinite(b) & (b != 0) & (a == 0)
    assert np.array_equal(np.signbit(q_rcp[zero]), np.signbit(a[zero]) ^ np.signbit(b[zero]))


def test_powf_quarter_matches_host_libm():
    rng = np.random.default_rng(3)
    bits = rng.integers(0x30000000, 0x45000000, 1_000_000, dtype=np.uint32)
    x = bits.view(np.float32).astype(np.float64)
    dev = vh.device_math(3, x)
    host = np.array([libm.powf(float(v), 0.25) for v in x.astype(np.float32)], dtype=np.float32).astype(np.float64)
    assert np.array_equal(dev, host), int((dev != host).sum())
