"""Checkpoint files on the host (no GPU): pg_ckpt_write_bs / pg_ckpt_read_bs and
pg_ckpt_write_pi_int / pg_ckpt_read_pi_int against files written by the reference's own code
(tests/golden/ckpt, made by tests/golden/make_ckpt_golden.py: save_bs_result,
src/engine/binary_splitting.cpp:48-71, and the pi_int writer, src/engine/pi_engine.cpp:494-506).
"""
import hashlib
import json
import os
import struct
import sys

import pytest

from helpers import GOLDEN, oracle, pkg

CKPT = os.path.join(GOLDEN, "ckpt")
sys.set_int_max_str_digits(0)
REF_FILES = {"bs_0_1419.ckpt": (0, 1419), "bs_1000_1419.ckpt": (1000, 1419), "bs_5_6.ckpt": (5, 6)}


@pytest.mark.parametrize("name", sorted(REF_FILES))
def test_read_reference_bs_files(name):
    a, b = REF_FILES[name]
    assert pkg.ckpt_read_bs(os.path.join(CKPT, name)) == oracle.bs(a, b)


@pytest.mark.parametrize("name", sorted(REF_FILES))
def test_write_matches_reference_bytes(name, tmp_path):
    a, b = REF_FILES[name]
    out = str(tmp_path / name)
    pkg.ckpt_write_bs(out, *oracle.bs(a, b))
    assert open(out, "rb").read() == open(os.path.join(CKPT, name), "rb").read()


def test_reference_bs_file_layout():
    """int sign, size_t count, count bytes (least significant first) for P, Q, R."""
    raw = open(os.path.join(CKPT, "bs_5_6.ckpt"), "rb").read()
    vals, off = [], 0
    for _ in range(3):
        sign, count = struct.unpack_from("<iQ", raw, off)
        off += 12
        vals.append(sign * int.from_bytes(raw[off:off + count], "little"))
        assert count == 0 or raw[off + count - 1] != 0  # no leading zero bytes
        off += count
    assert off == len(raw)
    assert tuple(vals) == oracle.bs(5, 6)


def test_pi_int_reference_file(tmp_path):
    src = os.path.join(CKPT, "pi_int_20000.ckpt")
    x = pkg.ckpt_read_pi_int(src)
    ref = open(os.path.join(GOLDEN, "pi_1000.txt")).read().strip()
    s = str(x)
    assert len(s) == 20001 and "3." + s[1:1001] == ref[:1002]
    out = str(tmp_path / "pi_int_20000.ckpt")
    pkg.ckpt_write_pi_int(out, x)
    assert open(out, "rb").read() == open(src, "rb").read()


def test_write_matches_reference_sha_at_1_5m_digits(tmp_path):
    """The reference program's root file at 1,500,000 digits (105,779 terms, 3.3 MB)."""
    g = json.load(open(os.path.join(GOLDEN, "ckpt_golden.json")))["1500000"]
    out = str(tmp_path / g["bs_file"])
    pkg.ckpt_write_bs(out, *oracle.bs(0, g["terms"]))
    assert os.path.getsize(out) == g["bs_bytes"]
    assert hashlib.sha256(open(out, "rb").read()).hexdigest() == g["bs_sha256"]


@pytest.mark.parametrize("vals", [(0, 1, 0), (1, 1, 1), (-1, 2**64, -(2**64 - 1)), (-(2**200 + 5), 3**100, 255),
                                  (2**63, -(2**127), 2**64 * 7)])
def test_round_trip_signs_and_limb_edges(vals, tmp_path):
    out = str(tmp_path / "x.ckpt")
    pkg.ckpt_write_bs(out, *vals)
    assert pkg.ckpt_read_bs(out) == vals
    # the byte count is the magnitude's significant bytes
    raw = open(out, "rb").read()
    count = struct.unpack_from("<iQ", raw, 0)[1]
    assert count == (abs(vals[0]).bit_length() + 7) // 8


def test_pi_int_zero_and_round_trip(tmp_path):
    out = str(tmp_path / "pi_int_1.ckpt")
    pkg.ckpt_write_pi_int(out, 0)
    assert open(out, "rb").read() == struct.pack("<Q", 0)
    assert pkg.ckpt_read_pi_int(out) == 0
    for x in (31, 2**64 - 1, 2**64, 10**5000 + 17):
        pkg.ckpt_write_pi_int(out, x)
        assert pkg.ckpt_read_pi_int(out) == x


def test_errors(tmp_path):
    with pytest.raises(pkg.PgError) as e:
        pkg.ckpt_read_bs(str(tmp_path / "missing.ckpt"))
    assert e.value.status == pkg.PG_ERR_IO
    good = open(os.path.join(CKPT, "bs_1000_1419.ckpt"), "rb").read()
    for cut in (3, 12, 100, len(good) - 1):  # short header, short data
        p = str(tmp_path / f"cut{cut}.ckpt")
        open(p, "wb").write(good[:cut])
        with pytest.raises(pkg.PgError) as e:
            pkg.ckpt_read_bs(p)
        assert e.value.status == pkg.PG_ERR_IO, cut
    # a count larger than the file
    p = str(tmp_path / "huge.ckpt")
    open(p, "wb").write(struct.pack("<iQ", 1, 1 << 60) + b"\x01" * 16)
    with pytest.raises(pkg.PgError) as e:
        pkg.ckpt_read_bs(p)
    assert e.value.status == pkg.PG_ERR_IO
    p = str(tmp_path / "pi.ckpt")
    open(p, "wb").write(struct.pack("<Q", 9) + b"\x01" * 8)
    with pytest.raises(pkg.PgError) as e:
        pkg.ckpt_read_pi_int(p)
    assert e.value.status == pkg.PG_ERR_IO
    with pytest.raises(pkg.PgError) as e:
        pkg.ckpt_write_pi_int(str(tmp_path / "no_such_dir" / "x.ckpt"), 5)
    assert e.value.status == pkg.PG_ERR_IO


def test_capacity_too_small_reports_need(tmp_path):
    import ctypes

    import numpy as np

    lib = pkg.load_library()
    path = os.path.join(CKPT, "bs_1000_1419.ckpt")
    n = (ctypes.c_size_t * 3)()
    sg = (ctypes.c_int * 3)()
    assert lib.pg_ckpt_read_bs(path.encode(), None, 0, n, sg) == pkg.PG_OK
    need = list(n)
    assert list(sg) == [-1, 1, -1]
    arrs = [np.zeros(4, dtype=np.uint64) for _ in range(3)]
    ptrs = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in arrs])
    assert lib.pg_ckpt_read_bs(path.encode(), ptrs, 4, n, sg) == pkg.PG_ERR_BAD_ARG
    assert list(n) == need
