"""CPU tests: pin the oracle against the reference's own known answers and golden fixtures.

Known-answer values are those of the reference's tests:
  tests/test_gmp_multiplier.cpp:30-125   products and squares
  tests/test_binary_splitting.cpp:16-126 terms_needed bounds, leaves k = 0, 1, 2, merge [0,2)
  tests/data/pi_1000.txt (via test_validation.cpp:48-72)
"""
import hashlib
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, oracle, pkg

L = pkg.int_to_limbs
I = pkg.limbs_to_int


def products(a, b):
    """All three oracle restatements plus Python's exact int product."""
    la, lb = L(a), L(b)
    return [I(oracle.mul_gmp(la, lb)), I(oracle.mul_schoolbook(la, lb)), I(oracle.mul_karatsuba(la, lb)),
            abs(a) * abs(b)]


@pytest.mark.parametrize(
    "a,b,expected",
    [
        (123, 456, 56088),                      # test_gmp_multiplier.cpp MultiplySmallNumbers
        (999999, 0, 0),                         # MultiplyByZero
        (42, 1, 42),                            # MultiplyByOne
        (7, 13, 91),                            # MultiplyNegativeNumbers (magnitudes; sign in the adaptor)
        (10**50, 10**50, 10**100),              # MultiplyLargeNumbers
        (12345, 12345, 152399025),              # SquareSmallNumber
        (10**500, 10**500, 10**1000),           # SquareLargeNumber
        (42, 42, 1764),                         # SquareNegativeNumber
    ],
)
def test_reference_product_kats(a, b, expected):
    for r in products(a, b):
        assert r == expected


def test_reference_large_operands_agree():
    # operands of test_gmp_multiplier.cpp:MultiplyVeryLargeNumbers and test_gpu_ntt_multiplier.cpp:89-114
    cases = [(2**3321, 3**2095), (2**3321 - 1, 3**2095 - 1), (2**33219 - 1, 3**20959 - 1),
             (123456789012345678901234567890, 987654321098765432109876543210)]
    for a, b in cases:
        rs = products(a, b)
        assert all(r == rs[-1] for r in rs)


@pytest.mark.parametrize("na,nb", [(1, 1), (1, 5), (5, 1), (31, 33), (64, 64), (100, 7), (257, 1000), (2000, 2000)])
def test_restatements_agree_random(na, nb):
    a = pkg.random_operand(na, 11 + na)
    b = pkg.random_operand(nb, 29 + nb)
    g = oracle.mul_gmp(a, b)
    assert np.array_equal(g, oracle.mul_karatsuba(a, b))
    assert I(g) == I(a) * I(b)
    if na * nb <= 200000:
        assert np.array_equal(g, oracle.mul_schoolbook(a, b))


def test_restatements_agree_all_ones():
    # long runs of 0xFFFF... limbs stress carry propagation
    for n in (1, 2, 17, 300):
        a = np.full(n, np.uint64(0xFFFFFFFFFFFFFFFF))
        assert I(oracle.mul_karatsuba(a, a)) == I(a) ** 2 == I(oracle.mul_gmp(a, a))


def test_product_golden_hashes_small():
    cases = json.load(open(os.path.join(GOLDEN, "products.json")))
    for c in cases:
        if c["na"] > 4096:
            continue
        a = pkg.random_operand(c["na"], c["seed"])
        b = a if c["nb"] == 0 else pkg.random_operand(c["nb"], c["seed"] + 7)
        r = oracle.mul_karatsuba(a, b)
        assert hashlib.sha256(r.astype("<u8").tobytes()).hexdigest() == c["sha256"]
        assert len(r) == c["len"]


def test_terms_needed_bounds():
    # test_binary_splitting.cpp:16-35
    t = oracle.terms_needed
    assert 8 <= t(100) <= 15
    assert 71 <= t(1000) <= 80
    assert 70000 <= t(1000000) <= 71000
    assert t(1_000_100) == 70_522      # 1M digits + 100 guard digits (pi_engine.cpp:214-218)
    assert t(100_000_100) == 7_051_375


def test_leaves_match_reference_tests():
    # test_binary_splitting.cpp:37-87
    assert oracle.bs(0, 1) == (1, 1, 13591409)
    assert oracle.bs(1, 2) == (-5, 10939058860032000, -2793657715)
    P, Q, _ = oracle.bs(2, 3)
    assert (P, Q) == (-231, 87512470880256000)
    P, Q, R = oracle.bs(0, 2)   # MergeTwoTerms
    assert P == -5 and Q == 10939058860032000 and R > 0


def test_oracle_bs_matches_reference_golden():
    g = json.load(open(os.path.join(GOLDEN, "bs_golden.json")))
    for key, (P, Q, R) in g["ranges"].items():
        a, b = map(int, key.split(","))
        assert oracle.bs(a, b) == (int(P, 16), int(Q, 16), int(R, 16)), key
    for key, hs in g["hash_ranges"].items():
        a, b = map(int, key.split(","))
        vals = oracle.bs(a, b)
        assert [hashlib.sha256(hex(v).encode()).hexdigest() for v in vals] == hs, key


def test_pi_1000_golden_is_pi():
    s = open(os.path.join(GOLDEN, "pi_1000.txt")).read()
    assert len(s) == 1002
    # test_validation.cpp:29-46 literals
    assert s.startswith("3.14159265358979323846264338327950288419716939937510"
                        "58209749445923078164062862089986280348253421170679")


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build not present")
def test_reference_build_reproduces_golden():
    assert oracle.ref_pi(1000) == open(os.path.join(GOLDEN, "pi_1000.txt")).read()
    assert oracle.ref_bs(0, 2) == oracle.bs(0, 2)
