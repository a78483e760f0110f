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


@pytest.mark.parametrize("wmin", ["1", "0"], ids=["wide", "narrow"])
@pytest.mark.parametrize("nd", [300_007, 2_000_000])
def test_to_decimal_both_configurations(eng, wmin, nd, monkeypatch):
    # the conversion's batched products (one shared power per level) in either configuration
    monkeypatch.setenv("PG_WIDE_MIN_LIMBS", wmin)
    x = rnd_bits(max(1, int(nd * 3.3219280948873623) - 2), nd + 1) % (10 ** nd)
    x = x - x % 10**40 + (10**40 - 1)  # a run of nines at the bottom: long carries
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


def _near_integer_root(m: int, digits: int, above_bits: int, below: bool, seed: int):
    """Q, R whose final-formula value V = 426880 sqrt(10005) Q 10^d / R lies within about
    2^-above_bits of the integer m: just above it (floor m) or, with below=True, just under it
    (floor m - 1). R = floor(S / m) (or + 1) with S = 426880 sqrt(10005) Q 10^d makes
    V - m = m frac(S / m) / R, so R's size sets how close V comes. Returns Q, R, floor(V) and
    the distance of V from m in bits (checked with exact integers)."""
    rng = np.random.default_rng(seed)
    rbits = m.bit_length() + above_bits
    qbits = rbits - (426880 * 100).bit_length() + 1
    q = int.from_bytes(rng.bytes((qbits + 7) // 8), "little") >> (8 * ((qbits + 7) // 8) - qbits)
    q |= 1 << (qbits - 1)
    base = 426880 * q * 10**digits
    r = math.isqrt(10005 * base * base) // m + (1 if below else 0)
    G = rbits + 64
    v_fix = math.isqrt(10005 * (base << G) ** 2) // r  # floor(V 2^G)
    fl = v_fix >> G
    dist = abs(v_fix - (m << G))  # |V - m| 2^G, to within one unit
    return q, r, fl, G - dist.bit_length()


@pytest.mark.parametrize("case", ["above", "below"])
def test_pi_finish_near_an_integer(eng, case):
    """Values within 2^-300 of an integer are closer than the first guard's error window: the
    formula must rerun with a larger guard and still return the exact floor (m, or m - 1 from
    just below), never a rounded one."""
    ref = open(os.path.join(GOLDEN, "pi_1000.txt")).read().strip()
    m = int(ref.replace(".", ""))
    q, r, fl, dbits = _near_integer_root(m, 1000, 300, case == "below", seed=7)
    assert 280 <= dbits <= 330  # the construction really lands near m
    want = m if case == "above" else m - 1
    assert fl == want
    s = str(want)
    assert eng.pi_finish(q, r, 1000) == s[0] + "." + s[1:]


def test_pi_finish_too_close_to_an_integer_fails_loudly(eng):
    """A value within 2^-1600 of an integer is beyond every guard the formula tries: it must
    report PG_ERR_INTERNAL rather than guess the floor."""
    ref = open(os.path.join(GOLDEN, "pi_1000.txt")).read().strip()
    m = int(ref.replace(".", ""))
    q, r, fl, dbits = _near_integer_root(m, 1000, 1600, False, seed=8)
    assert fl == m and dbits >= 1500
    with pytest.raises(pkg.PgError) as ei:
        eng.pi_finish(q, r, 1000)
    assert ei.value.status == pkg.PG_ERR_INTERNAL


@pytest.mark.parametrize("digits", [1, 10, 100, 999, 1000, 1001, 20_000])
def test_pg_pi_prefixes(eng, digits):
    ref = open(os.path.join(GOLDEN, "pi_1000.txt")).read().strip()
    got = eng.pi(digits).decode()
    assert len(got) == digits + 2
    if digits <= 1000:
        assert got == ref[: digits + 2]
    else:
        assert got[:1002] == ref


@pytest.mark.parametrize("digits", [1022, 1023, 1024, 2047, 2048, 2049, 4095, 70_001, 1_048_575, 1_048_577])
def test_pg_pi_tree_conversion_matches_exact_conversion(eng, digits, monkeypatch):
    """The digits come from the scaled remainder tree (a fraction of pi / 10 split by batched
    middle products, no division); with PG_EXACT_CONVERSION set they come from the exact final
    formula and divide-and-conquer conversion instead. Both must agree everywhere, at leaf and level
    boundaries of the tree included."""
    ref = open(os.path.join(GOLDEN, "pi_1000.txt")).read().strip()
    tree = eng.pi(digits)
    monkeypatch.setenv("PG_EXACT_CONVERSION", "1")
    exact = eng.pi(digits)
    assert tree == exact
    assert tree.decode()[:min(digits, 1000) + 2] == ref[:min(digits, 1000) + 2]


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
