"""GPU parity tests of the device-resident finish (pg_recip_floor, pg_sqrt_scaled,
pg_to_decimal, pg_pi_finish, pg_pi) through the C ABI.

The oracle for the quotient and root cores is exact integer arithmetic (Python ints: floor
division and math.isqrt), which is what the reference's mpf_div / mpf_sqrt approximate
(src/arithmetic/newton_divider.cpp:13-74; the reference's own tests only check short prefixes,
tests/test_newton_divider.cpp:29-136). The radix conversion is compared with Python's exact
int -> str (the role of mpz_get_str in src/io/base_converter.cpp). Digit strings are compared
with the reference program's committed outputs (tests/golden).
"""
import hashlib
import json
import math
import os
import sys

import numpy as np
import pytest

from helpers import GOLDEN, oracle, pkg

pytestmark = pytest.mark.gpu
sys.set_int_max_str_digits(0)


@pytest.fixture(scope="module")
def eng():
    e = pkg.Engine(0)
    yield e
    e.close()


def rnd_bits(bits: int, seed: int) -> int:
    n = (bits + 63) // 64
    x = pkg.limbs_to_int(pkg.random_operand(n, seed))
    x >>= 64 * n - bits
    return x | (1 << (bits - 1))


@pytest.mark.parametrize("bits", [1, 2, 63, 64, 65, 100, 129, 200, 1000, 4097, 65536, 1 << 20, 3 * (1 << 20) + 17])
def test_recip_floor_exact(eng, bits):
    for seed in range(3 if bits < 1 << 16 else 1):
        r = rnd_bits(bits, 31 * bits + seed)
        k = r.bit_length()
        assert eng.recip_floor(r) == (1 << (2 * k)) // r
    k = bits
    assert eng.recip_floor(1 << (k - 1)) == 1 << (k + 1)  # powers of two
    assert eng.recip_floor((1 << k) - 1) == (1 << (2 * k)) // ((1 << k) - 1)  # all ones


def mod_mersenne(x: int, n: int) -> int:
    """x mod 2^n - 1 by folding (Python's % would divide in quadratic time)."""
    m = (1 << n) - 1
    while x > m:
        x = (x & m) + (x >> n)
    return 0 if x == m else x


@pytest.mark.parametrize("logl", [6, 7, 10, 13, 14, 16])
def test_mul_wrap_is_the_product_modulo_2_32L_minus_1(eng, logl):
    L = 1 << logl
    M = (1 << (32 * L)) - 1
    half = L // 2
    full = [rnd_bits(64 * half, 7 * logl + i) for i in range(2)]
    cases = [(full[0], full[1]), (M, full[0]), (M, M), (1, 1), (1 << (32 * L - 1), 2), (0, full[1]),
             (rnd_bits(64, logl), full[1]), (M - 1, M - 1), (full[0], full[0])]
    for a, b in cases:
        got = eng.mul_wrap(a, b, logl)
        assert 0 <= got <= M, (logl, a.bit_length(), b.bit_length())
        assert mod_mersenne(got, 32 * L) == mod_mersenne(a * b, 32 * L), (logl, a.bit_length(), b.bit_length())


@pytest.mark.parametrize("s", [0, 1, 60, 64, 65, 200, 5000, 100_000, 1_000_003])
def test_sqrt_scaled_exact(eng, s):
    for a in (10005, 2, 3):
        assert eng.sqrt_scaled(a, s) == math.isqrt(a << (2 * s)), (a, s)


@pytest.mark.parametrize("nd", [1, 2, 19, 20, 127, 128, 129, 255, 256, 257, 1000, 4096, 10_001, 131_072, 300_007])
def test_to_decimal_matches_str(eng, nd):
    x = rnd_bits(max(1, int(nd * 3.3219280948873623) - 2), nd) % (10 ** nd)
    assert eng.to_decimal(x, nd) == str(x).zfill(nd)


def test_to_decimal_edges(eng):
    assert eng.to_decimal(0, 5) == "00000"
    assert eng.to_decimal(7, 300) == "0" * 299 + "7"
    nines = 10 ** 1000 - 1
    assert eng.to_decimal(nines, 1000) == "9" * 1000
    p = 10 ** 512
    assert eng.to_decimal(p, 513) == "1" + "0" * 512
    assert eng.to_decimal(p - 1, 513) == "0" + "9" * 512
    with pytest.raises(pkg.PgError):
        eng.to_decimal(10 ** 50, 10)


def test_pi_finish_from_oracle_series(eng):
    ref = open(os.path.join(GOLDEN, "pi_1000.txt")).read().strip()
    terms = oracle.terms_needed(1000)
    _, q, r = oracle.bs(0, terms)
    assert eng.pi_finish(q, r, 1000) == ref


@pytest.mark.parametrize("digits", [1, 10, 100, 999, 1000, 1001, 20_000])
def test_pg_pi_prefixes(eng, digits):
    ref = open(os.path.join(GOLDEN, "pi_1000.txt")).read().strip()
    got = eng.pi(digits).decode()
    assert len(got) == digits + 2
    if digits <= 1000:
        assert got == ref[: digits + 2]
    else:
        assert got[:1002] == ref


def test_pg_pi_repeated_and_interleaved_runs(eng):
    """Runs that repeat a digit count replay the splitting's captured CUDA graph; interleaving
    other counts (which reallocate its buffers) must never replay a stale graph."""
    ref = open(os.path.join(GOLDEN, "pi_1000.txt")).read().strip()
    first = eng.pi(30_000)
    assert first.decode()[:1002] == ref
    for d in (30_000, 30_000, 200, 30_000, 200_000, 30_000, 30_000):
        got = eng.pi(d)
        if d == 30_000:
            assert got == first
        else:
            assert got.decode()[:202] == ref[:202]


@pytest.mark.parametrize("digits", [1_000_000, 10_000_000, 100_000_000])
def test_pg_pi_matches_reference_hash(eng, digits):
    golden = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))[str(digits)]
    got = eng.pi(digits)
    assert len(got) == golden["bytes"]
    assert got[:66].decode() == golden["head"] and got[-64:].decode() == golden["tail"]
    assert hashlib.sha256(got).hexdigest() == golden["sha256"]
