"""Regenerate the golden fixtures in tests/golden/ from the reference build and the oracle.

Run from the repository root after `make -C oracle` (needs the reference sources mounted
for the reference build, at the directory named by the environment variable PI_REF; the
fixtures it writes are committed and used on machines without them):

    PI_REF=<reference checkout> python tests/golden/make_golden.py
    python tests/golden/make_golden.py --top     # only the top-size product hashes (products_top.json)

Outputs
  pi_1000.txt        "3." + 1000 digits from the reference program (checked byte-for-byte
                     against the reference's own tests/data/pi_1000.txt when it is mounted)
  pi_golden.json     sha256 / head / tail of the reference program's 1M, 10M and 100M digit files
                     (and 1B with --1b: `python tests/golden/make_golden.py --1b`)
  bs_golden.json     P, Q, R (hex) of the reference's BinarySplitting for small ranges, and
                     sha256 of P/Q/R for the 1M-digit term range
  products.json      sha256 of seeded random products computed by libgmp's mpz_mul
  products_top.json  the same for the largest products one transform takes (2^24-limb operands:
                     balanced, 3*2^23 x 2^23, 1:4, 1:16 and the square; about 10 s of mpz_mul each)
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from helpers import oracle, pkg  # noqa: E402

REF_DATA = os.path.join(os.environ.get("PI_REF", ""), "tests", "data", "pi_1000.txt")


def run_ref(digits: int, threads: int) -> bytes:
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "pi.txt")
        subprocess.run([oracle.PI_COMPUTE_REF, "--digits", str(digits), "--threads", str(threads), "--output", out],
                       check=True, stdout=subprocess.DEVNULL)
        return open(out, "rb").read()


def limb_hash(a) -> str:
    return hashlib.sha256(a.astype("<u8").tobytes()).hexdigest()


# Seeded product cases: (na, nb, seed). Shapes follow the multiply sweep: balanced,
# 1:4, 1:16 and squares, at sizes around transform-length boundaries.
PRODUCT_CASES = []
for n in [1, 2, 3, 7, 16, 31, 32, 33, 100, 1000, 1024, 1536, 4096, 6144, 16384, 65536, 98304, 262144, 1048576]:
    PRODUCT_CASES.append((n, n, 1000 + n))
    if n >= 4:
        PRODUCT_CASES.append((n, n // 4, 2000 + n))
    if n >= 16:
        PRODUCT_CASES.append((n, n // 16, 3000 + n))
    PRODUCT_CASES.append((n, 0, 4000 + n))  # nb == 0 encodes a square


# The largest products one transform takes (na + nb = 2^25 limbs, L = 2^26 points): the sizes the
# multiply's roofline is quoted on. (na, nb, seed), nb == 0 a square.
TOP_CASES = [(1 << 24, 1 << 24, 71), (3 << 23, 1 << 23, 72), (1 << 24, 1 << 22, 73), (1 << 24, 1 << 20, 74),
             (1 << 24, 0, 75)]


def product_entry(na: int, nb: int, seed: int) -> dict:
    a = pkg.random_operand(na, seed)
    r = oracle.mul_gmp(a, a) if nb == 0 else oracle.mul_gmp(a, pkg.random_operand(nb, seed + 7))
    return {"na": na, "nb": nb, "seed": seed, "len": int(len(r)), "sha256": limb_hash(r)}


def main_top() -> None:
    oracle.build()
    out = [product_entry(na, nb, seed) for na, nb, seed in TOP_CASES]
    json.dump(out, open(os.path.join(HERE, "products_top.json"), "w"), indent=1)
    print("top-size product hashes written to", HERE)


def main() -> None:
    if "--top" in sys.argv:
        main_top()
        return
    if not os.path.isdir(os.environ.get("PI_REF", "")):
        sys.exit("set PI_REF to the reference checkout (its tests/data/pi_1000.txt pins the reference build)")
    oracle.build()
    os.makedirs(HERE, exist_ok=True)

    pi1000 = run_ref(1000, 1)
    if os.path.exists(REF_DATA):
        assert pi1000 == open(REF_DATA, "rb").read().rstrip(b"\r\n "), "reference build disagrees with pi_1000.txt"
    open(os.path.join(HERE, "pi_1000.txt"), "wb").write(pi1000)

    path = os.path.join(HERE, "pi_golden.json")
    old = json.load(open(path)) if os.path.exists(path) else {}
    pig = {}
    # 1B digits (config 5) takes the reference ~15 minutes on 6 cores and 6.5 GB: only with --1b,
    # otherwise an earlier entry is kept
    sizes = [1_000_000, 10_000_000, 100_000_000] + ([1_000_000_000] if "--1b" in sys.argv else [])
    for d in sizes:
        s = run_ref(d, os.cpu_count() or 1)
        pig[str(d)] = {"sha256": hashlib.sha256(s).hexdigest(), "bytes": len(s), "head": s[:66].decode(),
                       "tail": s[-64:].decode()}
    if "1000000000" not in pig and "1000000000" in old:
        pig["1000000000"] = old["1000000000"]
    json.dump(pig, open(path, "w"), indent=1)

    bsg = {"ranges": {}, "hash_ranges": {}}
    for a, b in [(0, 1), (1, 2), (2, 3), (0, 2), (0, 8), (3, 11), (0, 79), (100, 357), (0, 1000)]:
        P, Q, R = oracle.ref_bs(a, b, 1)
        bsg["ranges"][f"{a},{b}"] = [hex(P), hex(Q), hex(R)]
    for a, b in [(0, 70522), (1000, 9000)]:
        P, Q, R = oracle.ref_bs(a, b, 1)
        bsg["hash_ranges"][f"{a},{b}"] = [hashlib.sha256(hex(v).encode()).hexdigest() for v in (P, Q, R)]
    json.dump(bsg, open(os.path.join(HERE, "bs_golden.json"), "w"), indent=1)

    prods = [product_entry(na, nb, seed) for na, nb, seed in PRODUCT_CASES]
    json.dump(prods, open(os.path.join(HERE, "products.json"), "w"), indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
