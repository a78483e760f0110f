"""Regenerate the checkpoint fixtures in tests/golden/ckpt/ from the reference build.

Run from the repository root after `make -C oracle` (needs the reference sources mounted for
the reference build; the fixtures it writes are committed and used on machines without them):

    python tests/golden/make_ckpt_golden.py

Every file here is written by the reference's own code, compiled unchanged:
  ckpt/bs_0_1419.ckpt, ckpt/pi_int_20000.ckpt
        the reference program run as `pi_compute --digits 20000 --checkpoint DIR`: the root
        splitting checkpoint that BinarySplitting::compute always saves
        (src/engine/binary_splitting.cpp:605-644) and the pi_int checkpoint of PiEngine
        (src/engine/pi_engine.cpp:494-506)
  ckpt/bs_1000_1419.ckpt, ckpt/bs_5_6.ckpt
        BinarySplitting::compute(a, b) with checkpointing enabled (ranges with a > 0, whose P
        and R are negative; bs_5_6 is a single leaf)
  ckpt_golden.json
        sha256 and sizes of the same program's files at 1,500,000 digits (105,779 terms: a
        root checkpoint of about 3.3 MB and a pi_int checkpoint of about 0.6 MB, too large to
        commit) and of its digit file
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from helpers import oracle  # noqa: E402

OUT = os.path.join(HERE, "ckpt")


def sha(path: str) -> str:
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def run_ref(digits: int, directory: str) -> str:
    out = os.path.join(directory, "pi.txt")
    subprocess.run([oracle.PI_COMPUTE_REF, "--digits", str(digits), "--threads", "8", "--checkpoint", directory,
                    "--output", out], check=True, stdout=subprocess.DEVNULL)
    return out


def main() -> None:
    oracle.build()
    if not oracle.ref_available():
        raise SystemExit("the reference build (oracle/_ref) is missing: run `make -C oracle` first")
    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        run_ref(20000, td)
        terms = oracle.terms_needed(20100)
        for name in (f"bs_0_{terms}.ckpt", "pi_int_20000.ckpt"):
            shutil.copy(os.path.join(td, name), os.path.join(OUT, name))
    with tempfile.TemporaryDirectory() as td:
        for a, b in ((1000, 1419), (5, 6)):
            shutil.copy(oracle.ref_bs_checkpoint(a, b, td), OUT)
    big = {}
    with tempfile.TemporaryDirectory() as td:
        digits = 1_500_000
        pi = run_ref(digits, td)
        terms = oracle.terms_needed(digits + 100)
        bs = os.path.join(td, f"bs_0_{terms}.ckpt")
        pint = os.path.join(td, f"pi_int_{digits}.ckpt")
        big[str(digits)] = {
            "terms": terms,
            "bs_file": os.path.basename(bs), "bs_bytes": os.path.getsize(bs), "bs_sha256": sha(bs),
            "pi_int_file": os.path.basename(pint), "pi_int_bytes": os.path.getsize(pint),
            "pi_int_sha256": sha(pint),
            "digits_bytes": os.path.getsize(pi), "digits_sha256": sha(pi),
            "files": sorted(os.listdir(td)),
        }
    json.dump(big, open(os.path.join(HERE, "ckpt_golden.json"), "w"), indent=1)
    print("wrote", sorted(os.listdir(OUT)), "and ckpt_golden.json")


if __name__ == "__main__":
    main()
