"""The two-word fixed-point split of the FP64 form's tile current (fx_split in
pic_internal.cuh), restated with the same IEEE operations on the host and
checked against exact rational arithmetic: s = v / q is exact (q a power of
two), s - rint(s) is exact, and the two words hold v to q * 2^-41; summed in
integers, n contributions stay within n * q * 2^-41 of the exact sum whatever
their order -- the property that keeps the plain form's current
order-independent and accurate where beam and return currents cancel."""
from fractions import Fraction

import numpy as np

LO = 40


def split(v, inv_q):
    s = v * inv_q                      # exact: inv_q is a power of two
    r = np.rint(s)                     # round half to even, as rint on the device
    d = s - r                          # exact (Sterbenz)
    il = np.rint(d * 2.0 ** LO)        # __double2ll_rn: round to nearest even
    return int(r), int(il), d


def test_split_is_exact_and_bounded():
    rng = np.random.default_rng(5)
    for e in (-53, -40, -10, 0, 20):
        inv_q = 2.0 ** (-e)
        q = Fraction(2) ** e
        v = rng.standard_normal(20000) * float(2.0 ** rng.integers(-30, 30)) * float(q) * 1e6
        for x in v[:4000]:
            ih, il, d = split(x, inv_q)
            s = Fraction(float(x)) / q
            assert Fraction(float(d)) == s - ih                      # the remainder is exact
            err = abs(s - (ih + Fraction(il, 2 ** LO)))
            assert err <= Fraction(1, 2 ** (LO + 1))                 # <= q 2^-41 in units of q


def test_integer_sums_are_order_independent_and_accurate():
    """Cancelling contributions (a beam current and a return current of
    opposite sign, 1e-9 of the bound): the two-word integer sum is the same
    in any order and within n q 2^-41 of the exact sum."""
    rng = np.random.default_rng(6)
    n = 5000
    beam = 4e-4 * (1 + 0.01 * rng.standard_normal(n))
    ret = -beam * (1 + 1e-9 * rng.standard_normal(n))
    v = np.concatenate([beam, ret])
    e = -53                                            # a tile bound of 320, as in the dense run
    inv_q, q = 2.0 ** (-e), Fraction(2) ** e
    exact = sum(Fraction(float(x)) for x in v)
    sums = []
    for perm in (np.arange(v.size), rng.permutation(v.size), rng.permutation(v.size)):
        hi = lo = 0
        for x in v[perm]:
            ih, il, _ = split(x, inv_q)
            hi += ih
            lo += il
        sums.append((hi, lo))
        total = (hi + Fraction(lo, 2 ** LO)) * q
        assert abs(total - exact) <= v.size * q / 2 ** (LO + 1)
    assert sums[0] == sums[1] == sums[2]
    # one word (the remainder dropped) is off by up to n q / 2 -- far more
    one_word = sum(split(x, inv_q)[0] for x in v) * q
    assert abs(one_word - exact) > 100 * v.size * q / 2 ** (LO + 1)


def lo32_bits(n):
    """fx_lo32_bits: L = 31 - bits(n), n < 2^bits(n)"""
    b = 0
    while (1 << b) <= n:
        b += 1
    return 31 - b


def split32(v, inv_q, L):
    s = v * inv_q
    r = np.rint(s)
    return int(r), int(np.rint((s - r) * 2.0 ** L))   # __double2int_rn


def test_lo32_bits_bound_every_sum():
    """A tile of n particles adds at most 2n times to one int32 word, each add
    at most 2^(L-1): the worst case (every add at the bound, one sign) stays
    below 2^31 for every n up to the two-word form's 2^23 limit, and the host's
    choice (L >= 14) covers tiles below 2^17 particles."""
    for n in list(range(1, 70000, 997)) + [2 ** k - 1 for k in range(1, 24)] + [2 ** k for k in range(1, 24)]:
        L = lo32_bits(n)
        assert L >= 7
        assert 2 * n * 2 ** (L - 1) < 2 ** 31
    assert lo32_bits(2 ** 17 - 1) == 14 and lo32_bits(2 ** 17) == 13
    # the c2 FP64 tile (4x4x16 cells, 3 x 32 particles per cell, 1.25 x + 64
    # capacity) takes the int32 word; the reference's default run (4x4x4
    # tiles of 4000 particles per cell) keeps the 64-bit one
    assert lo32_bits(int(256 * 96 * 1.25) + 3 * 64) >= 14
    assert lo32_bits(64 * 4000) < 14


def test_lo32_sums_are_order_independent_and_accurate():
    """The cancelling currents of the two-word test with an int32 second word
    at the resolution of a 2^15-particle tile: integer sums, so the same in
    any order, within n q 2^-(L+1) of the exact sum, and far inside the
    one-word error."""
    rng = np.random.default_rng(7)
    n = 5000
    beam = 4e-4 * (1 + 0.01 * rng.standard_normal(n))
    ret = -beam * (1 + 1e-9 * rng.standard_normal(n))
    v = np.concatenate([beam, ret])
    e = -53
    inv_q, q = 2.0 ** (-e), Fraction(2) ** e
    L = lo32_bits(2 ** 15)
    exact = sum(Fraction(float(x)) for x in v)
    sums = []
    for perm in (np.arange(v.size), rng.permutation(v.size)):
        hi = lo = 0
        for x in v[perm]:
            ih, il = split32(x, inv_q, L)
            assert abs(il) <= 2 ** (L - 1)
            hi += ih
            lo += il
        assert abs(lo) < 2 ** 31
        sums.append((hi, lo))
        total = (hi + Fraction(lo, 2 ** L)) * q
        assert abs(total - exact) <= v.size * q / 2 ** (L + 1)
    assert sums[0] == sums[1]
    one_word = sum(split32(x, inv_q, L)[0] for x in v) * q
    assert abs(one_word - exact) > 100 * v.size * q / 2 ** (L + 1)
