"""GPU parity tests of the multiply hot path through the C ABI (libpigpu.so).

Every product is compared bit-exactly with the oracle (libgmp's mpz_mul, the call the
reference's GmpMultiplier makes, gmp_multiplier.cpp:10-19) or with committed golden
hashes of oracle products, up to the largest products one transform takes (2^24-limb
operands, tests/golden/products_top.json).
Cases follow the reference's GPU suite (tests/test_gpu_ntt_multiplier.cpp:65-166) and
extend it with transform-length boundaries, uneven shapes, carry-chain stress and errors.
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, oracle, pkg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = pkg.Engine(0)
    yield e
    e.close()


def check(eng, a: np.ndarray, b: np.ndarray):
    got = eng.mul_limbs(a, b)
    exp = oracle.mul_gmp(a, b)
    assert len(got) == len(exp) and np.array_equal(got, exp), (len(a), len(b))


# ---------------------------------------------------------------- reference GPU suite cases
def test_reference_gpu_suite_cases(eng):
    G = pkg.limbs_to_int
    cases = [
        (12345, 67890),                                  # MultiplySmallNumbers
        (999999, 0),                                     # MultiplyByZero
        (123456789012345678901234567890, 1),             # MultiplyByOne
        (-12345, 67890),                                 # MultiplyNegative
        (2**3321 - 1, 3**2095 - 1),                      # Multiply1000DigitNumbers
        (2**33219 - 1, 3**20959 - 1),                    # Multiply10000DigitNumbers
        (2**332192 - 1, 3**209590 - 1),                  # Multiply100000DigitNumbers
    ]
    for a, b in cases:
        assert eng.mul(a, b) == a * b
    a = 2**33219 - 1
    assert eng.sqr(a) == a * a                           # SquareMatchesCpu
    del G


# ---------------------------------------------------------------- random sizes vs oracle
SIZES = [1, 2, 3, 4, 5, 7, 8, 15, 16, 17, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 255, 256, 511, 512,
         1000, 1023, 1024, 1025, 2047, 2048, 2049, 3000, 4095, 4096, 4097, 6144, 8191, 8192, 12288, 16384]


@pytest.mark.parametrize("n", SIZES)
def test_balanced_vs_oracle(eng, n):
    check(eng, pkg.random_operand(n, 100 + n), pkg.random_operand(n, 200 + n))


@pytest.mark.parametrize("n", [4, 16, 64, 100, 1024, 4096, 16384, 65536])
@pytest.mark.parametrize("ratio", [4, 16])
def test_unbalanced_vs_oracle(eng, n, ratio):
    a = pkg.random_operand(n, 300 + n)
    b = pkg.random_operand(max(1, n // ratio), 400 + n)
    check(eng, a, b)
    check(eng, b, a)


@pytest.mark.parametrize("n", [1, 2, 5, 64, 1000, 1024, 4096, 6144, 16384, 65536])
def test_square_vs_oracle(eng, n):
    a = pkg.random_operand(n, 500 + n)
    got = eng.sqr_limbs(a)
    assert np.array_equal(got, oracle.mul_gmp(a, a))
    assert np.array_equal(got, eng.mul_limbs(a, a))


def test_every_length_up_to_300(eng):
    # every transform length 2^6 .. 2^11 and every carry-block edge for small products
    for na in range(1, 301, 7):
        for nb in (1, 2, 3, na, 301 - na):
            check(eng, pkg.random_operand(na, na * 1000 + nb), pkg.random_operand(nb, nb * 1000 + na + 1))


# ---------------------------------------------------------------- carry stress and edge values
@pytest.mark.parametrize("n", [1, 3, 64, 1000, 4096, 70000])
def test_all_ones_operands(eng, n):
    ones = np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF))
    check(eng, ones, ones)
    check(eng, ones, ones[: max(1, n // 3)])
    one = np.array([1], dtype=np.uint64)
    check(eng, ones, one)


def test_powers_of_two_and_sparse(eng):
    for n in (1, 5, 300, 5000):
        a = np.zeros(n, dtype=np.uint64)
        a[-1] = np.uint64(1 << 63)
        check(eng, a, a)
        b = np.zeros(n, dtype=np.uint64)
        b[0] = 1
        b[-1] = 1
        check(eng, a, b)
        check(eng, b, b)


def test_leading_zero_limbs_are_trimmed(eng):
    a = np.array([5, 0, 0], dtype=np.uint64)
    b = np.array([7, 0], dtype=np.uint64)
    assert list(eng.mul_limbs(a, b)) == [35]
    assert len(eng.mul_limbs(np.zeros(4, dtype=np.uint64), b)) == 0
    assert len(eng.mul_limbs(np.zeros(0, dtype=np.uint64), b)) == 0


def test_output_may_alias_input(eng):
    lib = eng.lib
    a = pkg.random_operand(600, 77)
    b = pkg.random_operand(500, 78)
    exp = oracle.mul_gmp(a, b)
    buf = np.zeros(1100, dtype=np.uint64)
    buf[:600] = a
    n = ctypes.c_size_t(0)
    p = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    st = lib.pg_mul(eng.ctx, p, 600, b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), 500, p, 1100,
                    ctypes.byref(n))
    assert st == pkg.PG_OK
    assert np.array_equal(buf[: n.value], exp)


def test_errors_are_status_codes(eng):
    lib = eng.lib
    a = pkg.random_operand(10, 1)
    out = np.zeros(5, dtype=np.uint64)
    n = ctypes.c_size_t(0)
    P = ctypes.POINTER(ctypes.c_uint64)
    assert lib.pg_mul(eng.ctx, a.ctypes.data_as(P), 10, a.ctypes.data_as(P), 10, out.ctypes.data_as(P), 5,
                      ctypes.byref(n)) == pkg.PG_ERR_BAD_ARG
    assert "output buffer" in eng.last_error()
    big = (1 << 24) + 1
    z = np.zeros(big, dtype=np.uint64)  # buffer lengths above the limit are rejected before any read
    assert lib.pg_mul(eng.ctx, z.ctypes.data_as(P), big, z.ctypes.data_as(P), big, out.ctypes.data_as(P), 5,
                      ctypes.byref(n)) == pkg.PG_ERR_TOO_LARGE
    assert lib.pg_sqr(eng.ctx, z.ctypes.data_as(P), big, out.ctypes.data_as(P), 5,
                      ctypes.byref(n)) == pkg.PG_ERR_TOO_LARGE
    # the context stays usable
    check(eng, a, a)


# ---------------------------------------------------------------- golden hashes and large sizes
def test_golden_product_hashes(eng):
    for c in json.load(open(os.path.join(GOLDEN, "products.json"))):
        a = pkg.random_operand(c["na"], c["seed"])
        if c["nb"] == 0:
            r = eng.sqr_limbs(a)
        else:
            r = eng.mul_limbs(a, pkg.random_operand(c["nb"], c["seed"] + 7))
        assert len(r) == c["len"], c
        assert hashlib.sha256(r.astype("<u8").tobytes()).hexdigest() == c["sha256"], c


@pytest.mark.parametrize("logn", [20, 22])
def test_large_balanced_vs_oracle(eng, logn):
    n = 1 << logn
    check(eng, pkg.random_operand(n, 900 + logn), pkg.random_operand(n, 901 + logn))


TOP = json.load(open(os.path.join(GOLDEN, "products_top.json")))


@pytest.mark.parametrize("case", TOP, ids=[f"{c['na']}x{c['nb'] or 'sq'}" for c in TOP])
def test_max_size_products_bit_exact(eng, case):
    # the largest products one transform takes (na + nb = 2^25 limbs, L = 2^26 points), where the
    # roofline is quoted: compared word for word with mpz_mul through sha256 of the limbs
    a = pkg.random_operand(case["na"], case["seed"])
    if case["nb"] == 0:
        r = eng.sqr_limbs(a)
    else:
        r = eng.mul_limbs(a, pkg.random_operand(case["nb"], case["seed"] + 7))
    assert len(r) == case["len"]
    assert hashlib.sha256(r.astype("<u8").tobytes()).hexdigest() == case["sha256"]
