"""The rounding and exactness facts the evidence accumulation relies on, checked in numpy
float32/float64 arithmetic (round-to-nearest-even, as on the GPU)."""
import numpy as np


def kernel_units(v):
    v = np.maximum(np.float32(v), np.float32(0.0))
    m = np.float32(8388608.0)
    r = (v + m) - m  # float32 ops
    return np.where(v < m, r, v).astype(np.float64)


def test_magic_add_rounds_to_nearest_integer():
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.uniform(0, 2 ** 23, 200000), rng.uniform(0, 64, 200000),
                        np.arange(0, 64, 0.5), 2.0 ** rng.uniform(-30, 40, 100000)]).astype(np.float32)
    got = kernel_units(v)
    assert np.array_equal(got, np.rint(v.astype(np.float64)))
    assert np.all(got == np.floor(got))


def test_negative_values_clamp_to_zero():
    assert np.all(kernel_units(np.float32([-1e-3, -5.0, -1e12])) == 0.0)


def test_fp64_sums_of_units_are_order_independent():
    rng = np.random.default_rng(1)
    sigma_units = 2.0 ** 40  # largest kernel value in units
    v = np.float32(rng.uniform(0, 1, 2048) ** 3 * sigma_units)
    u = kernel_units(v)
    a = 0.0
    for x in u:
        a += x
    b = 0.0
    for x in u[::-1]:
        b += x
    c = 0.0
    for x in rng.permutation(u):
        c += x
    assert a == b == c == float(sum(int(x) for x in u))
