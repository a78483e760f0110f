"""Tests of the host engine (libpib200.so): binary splitting and pi digits.

CPU cases use GMP products (PIB_MODE_GMP) and check the engine against the reference's
known answers (tests/test_binary_splitting.cpp, tests/test_validation.cpp, tests/data/pi_1000.txt)
and the reference build's golden hashes. GPU cases route products through B200Multiplier
(PIB_MODE_PER_CALL, the per-call drop-in) and must give byte-identical digits.
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, oracle, pkg

GMP, PER_CALL, BATCHED = 0, 1, 2


@pytest.fixture(scope="module")
def lib():
    L = ctypes.CDLL(pkg.LIBPIB200)
    L.pib_pi.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.c_uint, ctypes.c_size_t, ctypes.c_int,
                         ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)]
    L.pib_pi.restype = ctypes.c_int
    P = ctypes.POINTER(ctypes.c_uint64)
    L.pib_bs.argtypes = [ctypes.c_ulong, ctypes.c_ulong, ctypes.c_int, ctypes.c_size_t, ctypes.c_int, P, P, P,
                         ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
    L.pib_bs.restype = ctypes.c_int
    L.pib_mul.argtypes = [P, ctypes.c_size_t, ctypes.c_int, P, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t,
                          ctypes.c_int, P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                          ctypes.POINTER(ctypes.c_int)]
    L.pib_mul.restype = ctypes.c_int
    L.pib_last_error.restype = ctypes.c_char_p
    return L


def drop_in_mul(lib, a, sa, b, sb, threshold=1):
    """a * b through pib_mul (pi::B200Multiplier::multiply on mpz_t); returns (limbs, sign)."""
    P = ctypes.POINTER(ctypes.c_uint64)
    cap = len(a) + len(b) + 1
    out = np.zeros(cap, dtype=np.uint64)
    n = ctypes.c_size_t()
    sg = ctypes.c_int()
    st = lib.pib_mul(a.ctypes.data_as(P), len(a), sa, b.ctypes.data_as(P), len(b), sb, threshold, 0,
                     out.ctypes.data_as(P), cap, ctypes.byref(n), ctypes.byref(sg))
    assert st == 0, lib.pib_last_error()
    return out[: n.value], sg.value


def pi_digits(lib, digits, mode, threshold=1024, threads=1):
    buf = ctypes.create_string_buffer(digits + 2)
    t = (ctypes.c_double * 8)()
    st = lib.pib_pi(digits, mode, threads, threshold, 0, buf, digits + 2, t)
    assert st == 0, lib.pib_last_error()
    return buf.raw[: digits + 2].decode(), list(t)


def bs(lib, a, b, mode, threshold=1):
    cap = 64 + 2 * (b - a) * 3 + 4 * (b - a)
    bufs = [np.zeros(cap, dtype=np.uint64) for _ in range(3)]
    ln = (ctypes.c_size_t * 3)()
    sg = (ctypes.c_int * 3)()
    P = ctypes.POINTER(ctypes.c_uint64)
    st = lib.pib_bs(a, b, mode, threshold, 0, *(x.ctypes.data_as(P) for x in bufs), cap, ln, sg)
    assert st == 0, lib.pib_last_error()
    return tuple(sg[i] * pkg.limbs_to_int(bufs[i][: ln[i]]) for i in range(3))


def test_engine_leaves_and_merges_gmp(lib):
    assert bs(lib, 0, 1, GMP) == (1, 1, 13591409)
    assert bs(lib, 1, 2, GMP) == (-5, 10939058860032000, -2793657715)
    assert bs(lib, 2, 3, GMP)[:2] == (-231, 87512470880256000)
    g = json.load(open(os.path.join(GOLDEN, "bs_golden.json")))
    for key, (P, Q, R) in g["ranges"].items():
        a, b = map(int, key.split(","))
        assert bs(lib, a, b, GMP) == (int(P, 16), int(Q, 16), int(R, 16)), key


def test_engine_digits_gmp(lib):
    # test_validation.cpp:29-89 and the reference program's 1000-digit file
    s50, _ = pi_digits(lib, 50, GMP)
    assert s50 == "3.14159265358979323846264338327950288419716939937510"
    s1000, t = pi_digits(lib, 1000, GMP)
    assert s1000 == open(os.path.join(GOLDEN, "pi_1000.txt")).read()
    assert t[3] > 0
    s100, _ = pi_digits(lib, 100, GMP)
    s500, _ = pi_digits(lib, 500, GMP)
    assert s1000.startswith(s500) and s500.startswith(s100)


def test_engine_1m_gmp_matches_reference_hash(lib):
    s, _ = pi_digits(lib, 1_000_000, GMP, threads=4)
    g = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["1000000"]
    assert hashlib.sha256(s.encode()).hexdigest() == g["sha256"]


def test_bad_mode_reports_error(lib):
    buf = ctypes.create_string_buffer(20)
    assert lib.pib_pi(10, 7, 1, 1, 0, buf, 20, None) != 0
    assert b"mode" in lib.pib_last_error()
    assert lib.pib_pi(10, GMP, 1, 1, 0, buf, 5, None) != 0


# ---------------------------------------------------------------- GPU: per-call drop-in
@pytest.mark.gpu
def test_per_call_bs_matches_oracle_with_every_product_on_gpu(lib):
    for a, b in [(0, 2), (0, 8), (3, 11), (0, 79), (100, 357), (0, 1000), (1000, 9000)]:
        assert bs(lib, a, b, PER_CALL, threshold=1) == oracle.bs(a, b), (a, b)


@pytest.mark.gpu
def test_per_call_digits_small_all_gpu(lib):
    s, _ = pi_digits(lib, 1000, PER_CALL, threshold=1)
    assert s == open(os.path.join(GOLDEN, "pi_1000.txt")).read()
    s, _ = pi_digits(lib, 10000, PER_CALL, threshold=1, threads=4)   # test_gpu_ntt_multiplier.cpp:159-166
    assert s.startswith("3.14159") and len(s) == 10002


@pytest.mark.gpu
def test_per_call_1m_digits_byte_identical(lib):
    # configuration 1: every product whose smaller operand has >= 2^10 limbs on the GPU, one call at a time
    s, t = pi_digits(lib, 1_000_000, PER_CALL, threshold=1024)
    g = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["1000000"]
    assert hashlib.sha256(s.encode()).hexdigest() == g["sha256"]


# ---------------------------------------------------------------- sign rule used by the device merges
def test_series_sign_rule_holds():
    # The device stores magnitudes: sgn P(a,b) = (-1)^(#terms k >= 1), Q > 0, sgn R(a,b) = sgn R(a,a+1),
    # and R = Qr*Rl + s*Pl*Rr with |Qr*Rl| > |Pl*Rr| (so the magnitude never changes sign).
    import random

    rnd = random.Random(5)
    ranges = [(0, 2), (0, 3), (1, 3), (0, 50), (7, 300)] + [(a, a + rnd.randint(2, 400)) for a in
                                                              (rnd.randint(0, 5000) for _ in range(30))]
    for a, b in ranges:
        m = a + (b - a) // 2
        Pl, Ql, Rl = oracle.bs(a, m)
        Pr, Qr, Rr = oracle.bs(m, b)
        P, Q, R = oracle.bs(a, b)
        neg = (b - a) - (1 if a == 0 else 0)
        assert (P < 0) == (neg % 2 == 1) and Q > 0
        assert (R > 0) == (a == 0)
        assert abs(Qr * Rl) > abs(Pl * Rr)
        s = (-1 if Rl < 0 else 1) * (-1 if Pl < 0 else 1) * (-1 if Rr < 0 else 1)
        e = (m - a) if a >= 1 else m
        assert s == (-1 if e % 2 else 1)
        assert abs(R) == abs(Qr * Rl) + s * abs(Pl * Rr)


# ---------------------------------------------------------------- GPU: level-batched device binary splitting
@pytest.mark.gpu
@pytest.mark.parametrize("a,b", [(0, 1), (1, 2), (5, 6), (0, 2), (0, 3), (1, 4), (0, 8), (3, 11), (0, 79),
                                 (100, 357), (0, 1000), (1000, 9000), (0, 4097), (12345, 31000)])
def test_batched_bs_matches_oracle(lib, a, b):
    assert bs(lib, a, b, BATCHED) == oracle.bs(a, b), (a, b)


@pytest.fixture(params=["1", "0"], ids=["wide", "narrow"])
def bs_config(request):
    """Every transform level of the splitting in the wide configuration (64-bit coefficients over
    five primes, PG_WIDE_MIN_LIMBS=1) or none of them (0); read whenever a range is planned."""
    old = os.environ.get("PG_WIDE_MIN_LIMBS")
    os.environ["PG_WIDE_MIN_LIMBS"] = request.param
    yield request.param
    if old is None:
        os.environ.pop("PG_WIDE_MIN_LIMBS", None)
    else:
        os.environ["PG_WIDE_MIN_LIMBS"] = old


@pytest.mark.gpu
@pytest.mark.parametrize("a,b", [(0, 79), (100, 357), (0, 1000), (1000, 9000), (0, 4097), (12345, 31000),
                                 (0, 70000)])
def test_batched_bs_both_configurations(lib, bs_config, a, b):
    # merges whose R^ subtracts (centred CRT lift) and adds both occur at every level
    assert bs(lib, a, b, BATCHED) == oracle.bs(a, b), (a, b, bs_config)


@pytest.mark.gpu
def test_batched_bs_golden_hash_1m_terms_both_configurations(lib, bs_config):
    g = json.load(open(os.path.join(GOLDEN, "bs_golden.json")))
    for key, hs in g["hash_ranges"].items():
        a, b = map(int, key.split(","))
        vals = bs(lib, a, b, BATCHED)
        assert [hashlib.sha256(hex(v).encode()).hexdigest() for v in vals] == hs, (key, bs_config)


@pytest.mark.gpu
def test_batched_bs_golden_hash_1m_terms(lib):
    g = json.load(open(os.path.join(GOLDEN, "bs_golden.json")))
    for key, hs in g["hash_ranges"].items():
        a, b = map(int, key.split(","))
        vals = bs(lib, a, b, BATCHED)
        assert [hashlib.sha256(hex(v).encode()).hexdigest() for v in vals] == hs, key


@pytest.mark.gpu
def test_batched_bs_repeated_range_replays_graph(lib):
    """The same range split three times: run directly, then captured into a CUDA graph, then
    replayed; every result equals the oracle's."""
    want = oracle.bs(0, 5000)
    for _ in range(3):
        assert bs(lib, 0, 5000, BATCHED) == want
    # a different range in between invalidates nothing it should not
    assert bs(lib, 100, 357, BATCHED) == oracle.bs(100, 357)
    assert bs(lib, 0, 5000, BATCHED) == want


@pytest.mark.gpu
def test_batched_digits_1000_and_1m(lib):
    s, _ = pi_digits(lib, 1000, BATCHED)
    assert s == open(os.path.join(GOLDEN, "pi_1000.txt")).read()
    s, _ = pi_digits(lib, 1_000_000, BATCHED)
    g = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["1000000"]
    assert hashlib.sha256(s.encode()).hexdigest() == g["sha256"]


@pytest.mark.gpu
def test_batched_digits_10m(lib):
    s, t = pi_digits(lib, 10_000_000, BATCHED)
    g = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["10000000"]
    assert hashlib.sha256(s.encode()).hexdigest() == g["sha256"]


BATCHED_HOST_FINISH = 4


@pytest.mark.gpu
def test_batched_host_finish_digits_1m(lib):
    """Batched splitting with the Newton finish on the host (B200 products) gives the same bytes."""
    s, _ = pi_digits(lib, 1000, BATCHED_HOST_FINISH)
    assert s == open(os.path.join(GOLDEN, "pi_1000.txt")).read()
    s, _ = pi_digits(lib, 1_000_000, BATCHED_HOST_FINISH)
    g = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["1000000"]
    assert hashlib.sha256(s.encode()).hexdigest() == g["sha256"]


# ---------------------------------------------------------------- Newton finish + D&C conversion (CPU)
GMP_NEWTON = 3


@pytest.mark.parametrize("digits", [1, 2, 3, 10, 50, 100, 999, 1000, 4096, 65537])
def test_newton_finish_matches_reference_digits_cpu(lib, digits):
    # integer Newton reciprocal / sqrt(10005) and divide-and-conquer decimal conversion (GMP products)
    s, _ = pi_digits(lib, digits, GMP_NEWTON)
    ref, _ = pi_digits(lib, digits, GMP)
    assert s == ref


def test_newton_finish_1m_cpu_hash(lib):
    s, _ = pi_digits(lib, 1_000_000, GMP_NEWTON, threads=8)
    g = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["1000000"]
    assert hashlib.sha256(s.encode()).hexdigest() == g["sha256"]


@pytest.mark.gpu
def test_drop_in_multiply_signs_and_routing(lib):
    a, b = pkg.random_operand(5000, 11), pkg.random_operand(4000, 12)
    for sa, sb in ((1, 1), (-1, 1), (1, -1), (-1, -1)):
        got, sg = drop_in_mul(lib, a, sa, b, sb)
        assert sg == sa * sb and np.array_equal(got, oracle.mul_gmp(a, b))
    got, sg = drop_in_mul(lib, a, 1, b, 1, threshold=10_000)  # routed to GMP below the threshold
    assert np.array_equal(got, oracle.mul_gmp(a, b))


@pytest.mark.gpu
def test_drop_in_multiply_beyond_one_transform(lib):
    """Products longer than pg_mul_max_limbs go through block products of pg_mul calls."""
    n = (1 << 25) - 5
    a, b = pkg.random_operand(n, 21), pkg.random_operand(12, 22)
    got, _ = drop_in_mul(lib, a, 1, b, 1)
    assert np.array_equal(got, oracle.mul_gmp(a, b))
    c = pkg.random_operand((1 << 24) + 3, 23)  # two blocks per operand: checked modulo three primes
    got, _ = drop_in_mul(lib, c, 1, c, 1)
    C, G = pkg.limbs_to_int(c), pkg.limbs_to_int(got)
    for q in (2**61 - 1, 1000000007, 998244353):
        assert (C % q) * (C % q) % q == G % q
