"""Host test of the Newton reciprocal's host base case (pi-compute_b200/csrc/host_div.h:
floor(2^e / v) by Knuth's Algorithm D in base 2^64) against Python's exact integer division, on
random divisors and on the carry-heavy shapes (all ones, a lone top bit plus one, alternating
words), at the sizes the reciprocal hands it (e = 2 * bits(v)) and at others. No GPU."""
import os
import random
import shutil
import subprocess

import pytest

from helpers import ROOT


def _limbs(x: int) -> list:
    out = []
    while x:
        out.append(x & (2**64 - 1))
        x >>= 64
    return out


@pytest.mark.skipif(not shutil.which("g++"), reason="needs g++")
def test_host_pow2_div_matches_exact_division(tmp_path):
    exe = str(tmp_path / "host_div_test")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "pi-compute_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "host_div_test.cpp"), "-o", exe], check=True)
    rng = random.Random(7)
    cases = []
    for bits in list(range(65, 300, 7)) + [1023, 1024, 1025, 4095, 4096, 4097, 8191, 16384, 16385, 24000]:
        v = rng.getrandbits(bits) | (1 << (bits - 1))
        cases.append((2 * bits, v))
        cases.append((2 * bits + rng.randrange(1, 200), v))
        cases.append((bits + rng.randrange(0, 64), v))
    for bits in (65, 128, 129, 4096, 16384):
        cases.append((2 * bits, (1 << bits) - 1))                      # all ones
        cases.append((2 * bits, (1 << (bits - 1)) + 1))                # a lone top bit, plus one
        cases.append((2 * bits, int("a" * (bits // 4), 16) | (1 << (bits - 1))))  # alternating bits
        cases.append((bits - 1, (1 << bits) - 1))                      # quotient 0
    inp = "".join(f"{e} {len(_limbs(v))} " + " ".join(f"{w:x}" for w in _limbs(v)) + "\n" for e, v in cases)
    r = subprocess.run([exe], input=inp, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.split("\n")
    for (e, v), line in zip(cases, lines):
        got = sum(int(w, 16) << (64 * i) for i, w in enumerate(line.split()))
        assert got == (1 << e) // v, (e, v.bit_length())
