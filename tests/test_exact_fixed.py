"""The exact prefix sums convert each float to 128-bit fixed point with 2^-80 resolution and each
prefix back to the nearest float (k3dom_b200/csrc/fixed128.cuh). The device forms the fixed-point
value in two 64-bit halves, and rounds back from the top 64 bits of the normalised value with the
bits below as a sticky bit, scaling by an add to the exponent field. This restates those steps in
Python integers and checks them against exact arithmetic: to_fixed(f) = floor(f 2^80) (0 for
negative, non-finite or >= 2^47 inputs), and from_fixed(v) = v 2^-80 rounded to the nearest float
(ties to even), over every exponent, including ties and sticky bits. CPU only."""
import struct

import numpy as np

M64 = (1 << 64) - 1
FRAC = 80


def f32_bits(x):
    return struct.unpack("<I", struct.pack("<f", float(np.float32(x))))[0]


def to_fixed_dev(x):
    b = f32_bits(x)
    if b >= 0x7F800000:
        return 0
    e, frac = b >> 23, b & 0x7FFFFF
    m = (frac | 0x800000) if e else frac
    sh = (e if e else 1) - 150 + FRAC
    if sh < 0:
        return m >> min(-sh, 63)
    if sh > 127 - 24:
        return 0
    if sh < 64:
        lo = (m << sh) & M64
        hi = m >> (64 - sh) if sh > 40 else 0
    else:
        lo, hi = 0, m << (sh - 64)
    return (hi << 64) | lo


def round_int_to_f32(x):
    """Nearest float32 to the non-negative integer x (ties to even), as a Python float."""
    n = x.bit_length()
    if n <= 24:
        return float(x)
    s = n - 24
    q, rem, half = x >> s, x & ((1 << s) - 1), 1 << (s - 1)
    if rem > half or (rem == half and q & 1):
        q += 1
    return float(q) * 2.0 ** s


def from_fixed_dev(v):
    hi, lo = v >> 64, v & M64
    if hi == 0:
        if lo == 0:
            return 0.0
        f, k = round_int_to_f32(lo), -FRAC
    else:
        s = 64 - hi.bit_length()
        top = (((hi << s) | (lo >> (64 - s))) & M64) if s else hi
        rest = ((lo << s) & M64) if s else lo
        f, k = round_int_to_f32(top | (1 if rest else 0)), 64 - s - FRAC
    return f * 2.0 ** k  # the exponent add: exact for a normal result


def test_to_fixed_is_the_floor_of_the_scaled_value():
    rng = np.random.default_rng(3)
    xs = list(np.float32(2.0 ** rng.uniform(-100, 50, 4000)))
    xs += [np.float32(v) for v in (0.0, 1.0, 2.0 ** 46, np.nextafter(np.float32(2.0 ** 47), np.float32(0)),
                                   2.0 ** 47, 1e-40, 2.0 ** -80, 2.0 ** -81, 3.0 * 2.0 ** -82)]
    for x in xs:
        # a float32 times 2^80 is exact in FP64, and int() of an exact FP64 integer is exact
        want = int(np.floor(float(x) * 2.0 ** FRAC)) if float(x) < 2.0 ** 47 else 0
        assert to_fixed_dev(x) == want, x
    for bad in (-1.0, -0.0, float("inf"), float("nan"), 1e30):
        assert to_fixed_dev(bad) == 0


def test_from_fixed_rounds_to_nearest_even():
    rng = np.random.default_rng(4)
    vals = []
    for bits in range(1, 128):
        for _ in range(20):
            vals.append(int(rng.integers(0, 1 << 62)) << max(0, bits - 62) | (1 << (bits - 1)))
        if bits > 25:  # exact ties, with and without a sticky bit below, odd and even significands
            s = bits - 24
            for q in ((1 << 23) | 1, (1 << 23) | 2, (1 << 24) - 1):
                vals += [(q << s) | (1 << (s - 1)), (q << s) | (1 << (s - 1)) | (1 if s > 1 else 0)]
    for v in vals:
        v &= (1 << 127) - 1
        want = round_int_to_f32(v) * 2.0 ** -FRAC if v else 0.0
        got = from_fixed_dev(v)
        assert got == want, (hex(v), got, want)
        assert got == float(np.float32(got))  # a float32 value


def test_round_trip_of_prefix_sums():
    rng = np.random.default_rng(5)
    w = np.float32(rng.uniform(0, 1, 3000) ** 4)
    acc = 0
    for x in w:
        acc += to_fixed_dev(x)
        assert from_fixed_dev(acc) == round_int_to_f32(acc) * 2.0 ** -FRAC
    assert acc == sum(to_fixed_dev(x) for x in w[::-1])
