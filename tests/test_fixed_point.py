"""The mixed engine's fixed-point deposit arithmetic, restated in numpy FP32.

The push kernel (felis_b200/csrc/lib/k_batch.cu, `fix` and `quantum`) rounds
each deposit term v / q to an integer by one FP32 add of 1.5 * 2^23 to the
exact product v * (1/q), reading the integer from the low mantissa bits.  These
checks pin that identity against round-half-even over the whole range the
kernel allows (|v / q| < 2^22), and the quantum rule that keeps every term in
that range and every sum below 2^30 quanta.
"""
import math

import numpy as np

MAGIC = np.float32(12582912.0)  # 1.5 * 2^23
MAGIC_BITS = np.int32(0x4B400000)
ACC_BITS = 31


def fix(v: np.ndarray, inv_q: np.float32) -> np.ndarray:
    """The kernel's rounding: (v * inv_q) exact in FP32, one rounded add."""
    y = (v.astype(np.float32) * np.float32(inv_q)).astype(np.float32)
    return ((y + MAGIC).astype(np.float32).view(np.int32) - MAGIC_BITS).astype(np.int64)


def quantum(bound: float, term: float) -> float:
    """The kernel's quantum 2^e: bound / q < 2^(ACC_BITS - 1), term / q < 2^22."""
    if not bound > 0.0:
        return 1.0
    e = math.frexp(bound)[1] - 1 + 2 - ACC_BITS  # ilogb(bound) + 2 - ACC_BITS
    if term > 0.0:
        e = max(e, math.frexp(term)[1] - 1 - 21)
    return math.ldexp(1.0, max(e, -120))


def test_shift_rounding_equals_round_half_even():
    rng = np.random.default_rng(7)
    lim = 2.0**22
    y = np.concatenate([
        rng.uniform(-lim, lim, 400000),
        rng.uniform(-64.0, 64.0, 200000),
        np.arange(-1000, 1000) + 0.5,  # ties: to even
        np.array([0.0, -0.0, 0.49999997, -0.49999997, 1.5, -1.5, 2.5, -2.5, lim - 1.0, -lim, -lim + 0.5]),
    ]).astype(np.float32)
    got = fix(y, np.float32(1.0))
    want = np.rint(y.astype(np.float64)).astype(np.int64)
    assert np.array_equal(got, want)


def test_shift_rounding_with_power_of_two_quanta():
    rng = np.random.default_rng(8)
    for e in (-60, -30, -7, 0, 5, 20):
        inv_q = np.float32(2.0**-e)
        v = (rng.uniform(-1.0, 1.0, 100000) * 2.0**(e + 21)).astype(np.float32)
        got = fix(v, inv_q)
        want = np.rint(v.astype(np.float64) * 2.0**-e).astype(np.int64)
        assert np.array_equal(got, want), e


def test_quantum_keeps_terms_and_sums_in_range():
    rng = np.random.default_rng(9)
    for _ in range(2000):
        term = float(np.float32(10.0 ** rng.uniform(-12, 6)))
        count = int(rng.integers(1, 1 << 16))
        bound = term * count
        q = quantum(bound, term)
        assert term / q < 2.0**22
        assert bound / q < 2.0**30
        # a slice of many particles keeps the precision the sum bound alone gives
        if count >= 1024:
            assert q == quantum(bound, 0.0)


def test_sums_of_rounded_terms_stay_in_int32():
    rng = np.random.default_rng(10)
    count, term = 8192, 3.7e-9
    q = quantum(term * count * 1.0625, term * 1.0625)
    v = rng.uniform(-term, term, count).astype(np.float32)
    s = int(fix(v, np.float32(1.0 / q)).sum())
    assert abs(s) < 2**31
    assert abs(s * q - float(v.astype(np.float64).sum())) <= count * q / 2
