"""The drop-in inside the reference's own code: the reference's UNCHANGED BinarySplitting and
PiEngine (compiled from its sources into oracle/_ref/libpiref_b200.so) run with the library's
pi::B200Multiplier behind their `Multiplier&` (binary_splitting.h:39, pi_engine.h:34), the way the
reference's main.cpp:128-176 hands them its own GPU multipliers. P/Q/R must equal the reference's
golden values (written by its GmpMultiplier run, tests/golden/bs_golden.json) and the digits its
golden file hashes, with products of at least `threshold` limbs on the B200 (1: every product;
1024: the per-call configuration).
"""
import hashlib
import json
import os

import pytest

from helpers import GOLDEN, oracle

pytestmark = pytest.mark.gpu

needs_shim = pytest.mark.skipif(not os.path.exists(oracle.LIBPIREF_B200),
                                reason="oracle/_ref/libpiref_b200.so not built (needs the reference sources)")


@needs_shim
@pytest.mark.parametrize("threshold", [1, 1024])
def test_reference_binary_splitting_with_b200_multiplier(threshold):
    g = json.load(open(os.path.join(GOLDEN, "bs_golden.json")))
    calls = 0
    for key, (P, Q, R) in g["ranges"].items():
        a, b = map(int, key.split(","))
        p, q, r, c = oracle.refb_bs(a, b, threshold, threads=4)
        calls += c
        assert (p, q, r) == (int(P, 16), int(Q, 16), int(R, 16)), key
    for key, hashes in g["hash_ranges"].items():
        a, b = map(int, key.split(","))
        if threshold == 1 and b - a > 10000:
            continue  # every one of ~280k products one call at a time: the 1M-digit range runs at 1024
        p, q, r, c = oracle.refb_bs(a, b, threshold, threads=4)
        calls += c
        assert [hashlib.sha256(hex(v).encode()).hexdigest() for v in (p, q, r)] == hashes, key
    assert calls > 0  # the B200 computed products (threshold 1: all of them)


@needs_shim
def test_reference_pi_engine_with_b200_multiplier_1m_digits():
    want = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["1000000"]["sha256"]
    digits, calls = oracle.refb_pi(1_000_000, threshold=1024, threads=8)
    assert calls > 100
    assert hashlib.sha256(digits.encode()).hexdigest() == want
