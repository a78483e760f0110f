"""GPU tests of the paths for numbers beyond one transform: block products (DevArith products
longer than the longest transform) and splitting trees cut into level-batched subtrees merged on
the device. At full size they only run for pi beyond ~300M digits; PG_MAX_LOGL lowers the
longest transform for one process, so the same code runs here at small sizes and is checked
against the oracle (libgmp through oracle/, Python integers) and the reference's digit hashes.
"""
import hashlib
import json
import os
import subprocess
import sys

import pytest

from helpers import GOLDEN, ROOT, pkg

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import math, os, sys
sys.set_int_max_str_digits(0)
sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
from helpers import oracle, pkg

def rnd_bits(bits, seed):
    n = (bits + 63) // 64
    x = pkg.limbs_to_int(pkg.random_operand(n, seed)) >> (64 * n - bits)
    return x | (1 << (bits - 1))

with pkg.Engine(0) as eng:
    for a, b in ((0, 3000), (1000, 9000), (0, 20000), (12345, 16001)):
        assert eng.bs(a, b) == oracle.bs(a, b), (a, b)
    for bits in (70_000, 333_333):
        r = rnd_bits(bits, bits)
        assert eng.recip_floor(r) == (1 << (2 * r.bit_length())) // r, bits
    for s in (150_000, 400_001):
        assert eng.sqrt_scaled(10005, s) == math.isqrt(10005 << (2 * s)), s
    for nd in (40_000, 250_001):
        x = rnd_bits(int(nd * 3.3219280948873623) - 2, nd) % (10 ** nd)
        assert eng.to_decimal(x, nd) == str(x).zfill(nd), nd
print("ok")
"""


def test_block_products_and_split_trees_under_a_lowered_cap():
    env = dict(os.environ, PG_MAX_LOGL="12")
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-4000:]


@pytest.mark.parametrize("cap", ["14", "17"])
def test_pi_1m_digits_with_a_lowered_cap_matches_reference(tmp_path, cap):
    golden = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["1000000"]
    out = str(tmp_path / "pi.txt")
    env = dict(os.environ, PG_MAX_LOGL=cap)
    subprocess.run([pkg.PI_B200_BIN, "--batched", "--digits", "1000000", "--output", out], env=env, check=True,
                   stdout=subprocess.DEVNULL, timeout=600)
    assert hashlib.sha256(open(out, "rb").read()).hexdigest() == golden["sha256"]


def test_pi_1b_digits_matches_reference():
    """Config 5: a billion digits through the split tree and block products at full size. The
    first 100M digits must equal the 100M run's; the whole file the reference program's 1B run."""
    g = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))
    eng = pkg.Engine(0)
    try:
        got = eng.pi(1_000_000_000)
    finally:
        eng.close()
    assert len(got) == 1_000_000_002
    assert hashlib.sha256(got[:100_000_002]).hexdigest() == g["100000000"]["sha256"]
    want = g["1000000000"]
    assert got[:66].decode() == want["head"] and got[-64:].decode() == want["tail"]
    assert hashlib.sha256(got).hexdigest() == want["sha256"]


ADD_SCRIPT = r"""
import math, os, sys
sys.set_int_max_str_digits(0)
sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
from helpers import pkg

with pkg.Engine(0) as eng:
    # long runs of ones and zeros: sums whose carries cross many 2048-limb segments
    for k in (3 * (1 << 20) + 17, 1 << 21):
        for r in ((1 << k) - 1, (1 << (k - 1)) + 1, ((1 << k) - 1) ^ (1 << (k // 2))):
            assert eng.recip_floor(r) == (1 << (2 * r.bit_length())) // r, (k, r.bit_length())
    s = 400_001
    assert eng.sqrt_scaled(10005, s) == math.isqrt(10005 << (2 * s)), s
    print(eng.pi(1_000_000)[-64:].decode())
print("ok")
"""


@pytest.mark.parametrize("onepass", ["1", "0"])
def test_long_sums_one_pass_and_three_launch_forms(onepass):
    """Plain sums of long numbers run as one launch with a bounded look-back between segments
    (default) or as three launches (PG_ADD_ONEPASS=0); both give exact quotients and roots where
    the carries run across many segments, and the same pi digits."""
    env = dict(os.environ, PG_ADD_ONEPASS=onepass)
    r = subprocess.run([sys.executable, "-c", ADD_SCRIPT, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-4000:]
    golden = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["1000000"]
    assert r.stdout.strip().splitlines()[-2] == golden["tail"]
