"""GPU parity of both transform configurations the product chooses between:

* 32-bit coefficients over three primes < 2^31 (transforms of 2^26 points at most);
* the wide configuration, 64-bit coefficients (one per limb) over five primes < 2^31 whose product
  ~2^153.4 bounds every coefficient of a product of up to 2^25 limbs (min(na, nb) (2^64 - 1)^2 <
  q0 ... q4): half the transform length, 5/6 of the residue work per product bit.

A product of at least PG_WIDE_MIN_LIMBS limbs (na + nb) runs wide (the library's default threshold
is 2^13; the variable is read on every call). Each case runs with the boundary at 1 (every product
wide) and at 0 (none), bit-exact against the oracle (libgmp's mpz_mul, the reference's
GmpMultiplier call) and against each other. The reference multiplies with one fixed setting
(three primes, 15-bit digits, int_ntt.h:30-42).
"""
import os

import numpy as np
import pytest

from helpers import oracle, pkg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = pkg.Engine(0)
    yield e
    e.close()


@pytest.fixture(params=["1", "0"], ids=["wide", "narrow"])
def config(request):
    old = os.environ.get("PG_WIDE_MIN_LIMBS")
    os.environ["PG_WIDE_MIN_LIMBS"] = request.param
    yield request.param
    if old is None:
        os.environ.pop("PG_WIDE_MIN_LIMBS", None)
    else:
        os.environ["PG_WIDE_MIN_LIMBS"] = old


SIZES = [(1, 1), (1, 2), (2, 2), (3, 5), (31, 33), (32, 32), (33, 31), (100, 37), (511, 513), (1000, 24), (2048, 2048),
         (3000, 1096), (4096, 4095), (6000, 2193), (8192, 8192), (12288, 4096), (1 << 15, 1 << 15), (100000, 31000),
         (1 << 17, 1 << 15)]


@pytest.mark.parametrize("na,nb", SIZES)
def test_products_vs_oracle(eng, config, na, nb):
    a = pkg.random_operand(na, 17 * na + nb)
    b = pkg.random_operand(nb, 19 * nb + na)
    exp = oracle.mul_gmp(a, b)
    assert np.array_equal(eng.mul_limbs(a, b), exp)
    assert np.array_equal(eng.mul_limbs(b, a), exp)


@pytest.mark.parametrize("n", [1, 2, 7, 64, 1000, 4096, 9000, 1 << 16])
def test_squares_and_carry_stress(eng, config, n):
    a = pkg.random_operand(n, 23 * n)
    assert np.array_equal(eng.sqr_limbs(a), oracle.mul_gmp(a, a))
    ones = np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF))  # the largest coefficients the bound admits
    assert np.array_equal(eng.mul_limbs(ones, ones), oracle.mul_gmp(ones, ones))
    assert np.array_equal(eng.sqr_limbs(ones), oracle.mul_gmp(ones, ones))


def test_every_wide_length_boundary(eng, config):
    # na + nb - 1 coefficients around each power of two from 2^6 to 2^16 (the wide transform length)
    for l in range(6, 17):
        for s in (-1, 0, 1, 2):
            tot = (1 << l) + s
            na = max(1, tot // 3)
            nb = max(1, tot - na)
            a, b = pkg.random_operand(na, l * 10 + s + 5), pkg.random_operand(nb, l * 10 + s + 6)
            assert np.array_equal(eng.mul_limbs(a, b), oracle.mul_gmp(a, b)), (na, nb)


R3_SIZES = [(6000, 6000), (4097, 8000), (3 << 14, 3 << 14), (100000, 90000), (150000, 3000), (1 << 17, 1 << 16),
            (3 << 19, (3 << 19) - 5)]


@pytest.mark.parametrize("na,nb", R3_SIZES)
def test_three_times_power_of_two_lengths(eng, na, nb, monkeypatch):
    """Wide products whose na + nb - 1 coefficients fit 3 * 2^m points (3/4 of the next power of
    two) run a radix-3 step plus 2^m-point passes (the transform's roots have order 3 * 2^25);
    PG_RADIX3=0 sends the same product through the power-of-two length. Both bit-exact against
    the oracle, squares and all-ones operands (the largest coefficients) included."""
    monkeypatch.setenv("PG_WIDE_MIN_LIMBS", "1")
    monkeypatch.setenv("PG_RADIX3", "12")  # from 3 * 2^12 points (the default starts at 3 * 2^20)
    a = pkg.random_operand(na, 29 * na + nb)
    b = pkg.random_operand(nb, 31 * nb + na)
    exp = oracle.mul_gmp(a, b)
    assert np.array_equal(eng.mul_limbs(a, b), exp)
    monkeypatch.setenv("PG_RADIX3", "0")
    assert np.array_equal(eng.mul_limbs(a, b), exp)
    monkeypatch.setenv("PG_RADIX3", "12")
    assert np.array_equal(eng.sqr_limbs(a), oracle.mul_gmp(a, a))
    ones = np.full(na, np.uint64(0xFFFFFFFFFFFFFFFF))
    assert np.array_equal(eng.mul_limbs(ones, b), oracle.mul_gmp(ones, b))
