"""GPU tests of the checkpointed device pipeline (pg_bs_checkpointed, pg_pi_checkpointed and the
CLI's --checkpoint): the files it writes are byte-identical to the reference's own
(tests/golden/ckpt, tests/golden/ckpt_golden.json), files written by the reference resume it,
and partial trees of node files are merged on the device into the same digits. The resume rules
follow BinarySplitting::compute / compute_parallel / compute_sequential and save_checkpoint
(src/engine/binary_splitting.cpp:104-135, 295-302, 350-360, 605-644) and PiEngine's pi_int
file (src/engine/pi_engine.cpp:263-284, 494-506).
"""
import hashlib
import json
import os
import shutil
import subprocess
import sys

import pytest

from helpers import GOLDEN, oracle, pkg

pytestmark = pytest.mark.gpu
sys.set_int_max_str_digits(0)
CKPT = os.path.join(GOLDEN, "ckpt")
PI1000 = open(os.path.join(GOLDEN, "pi_1000.txt")).read().strip()


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def same_file(a, b):
    return open(a, "rb").read() == open(b, "rb").read()


def pi_from_pi_int_file(path):
    s = str(pkg.ckpt_read_pi_int(path))
    return "3." + s[1:]


@pytest.fixture(scope="module")
def eng():
    e = pkg.Engine(0)
    yield e
    e.close()


def test_fresh_run_writes_the_reference_files(eng, tmp_path):
    d = str(tmp_path / "ck")  # created by the call
    got, rep = eng.pi_checkpointed(20000, d)
    assert sorted(os.listdir(d)) == ["bs_0_1419.ckpt", "pi_int_20000.ckpt"]
    for name in os.listdir(d):
        assert same_file(os.path.join(d, name), os.path.join(CKPT, name)), name
    assert rep == {"root_loaded": 0, "root_saved": 1, "pi_int_loaded": 0, "pi_int_saved": 1, "nodes_loaded": 0,
                   "subtrees_computed": 1, "merges": 0}
    assert got.decode() == pi_from_pi_int_file(os.path.join(CKPT, "pi_int_20000.ckpt"))
    assert got.decode()[:1002] == PI1000
    assert got == eng.pi(20000)


def test_resume_from_reference_files(eng, tmp_path):
    want = pi_from_pi_int_file(os.path.join(CKPT, "pi_int_20000.ckpt"))
    # both files: the splitting and the final formula are skipped
    d = str(tmp_path / "both")
    os.makedirs(d)
    for name in ("bs_0_1419.ckpt", "pi_int_20000.ckpt"):
        shutil.copy(os.path.join(CKPT, name), d)
    got, rep = eng.pi_checkpointed(20000, d)
    assert got.decode() == want
    assert rep["root_loaded"] == 1 and rep["pi_int_loaded"] == 1 and rep["subtrees_computed"] == 0
    assert rep["root_saved"] == 0 and rep["pi_int_saved"] == 0
    # only the splitting file: the final formula runs and writes pi_int
    d = str(tmp_path / "bs_only")
    os.makedirs(d)
    shutil.copy(os.path.join(CKPT, "bs_0_1419.ckpt"), d)
    got, rep = eng.pi_checkpointed(20000, d)
    assert got.decode() == want and rep["root_loaded"] == 1 and rep["pi_int_saved"] == 1
    assert same_file(os.path.join(d, "pi_int_20000.ckpt"), os.path.join(CKPT, "pi_int_20000.ckpt"))


def test_partial_tree_merged_on_device(eng, tmp_path):
    """Node files for [0, 709) and [1064, 1419) of the 1419-term tree (split points 709, 1064):
    [709, 1064) is one device splitting, two merges rebuild the root. A file on a range that is
    not a node is ignored; a truncated node file counts as absent."""
    d = str(tmp_path / "partial")
    os.makedirs(d)
    for a, b in ((0, 709), (1064, 1419)):
        pkg.ckpt_write_bs(os.path.join(d, f"bs_{a}_{b}.ckpt"), *oracle.bs(a, b))
    pkg.ckpt_write_bs(os.path.join(d, "bs_3_17.ckpt"), 1, 1, 1)  # not a node of this tree: unused
    raw = open(os.path.join(d, "bs_0_709.ckpt"), "rb").read()
    open(os.path.join(d, "bs_709_1064.ckpt"), "wb").write(raw[:50])  # a node, but short: recomputed
    got, rep = eng.pi_checkpointed(20000, d)
    assert got.decode() == pi_from_pi_int_file(os.path.join(CKPT, "pi_int_20000.ckpt"))
    assert rep["nodes_loaded"] == 2 and rep["subtrees_computed"] == 1 and rep["merges"] == 2
    assert rep["root_saved"] == 1 and rep["root_loaded"] == 0
    assert same_file(os.path.join(d, "bs_0_1419.ckpt"), os.path.join(CKPT, "bs_0_1419.ckpt"))
    # the root's two children are removed (bs_709_1419 never existed); deeper files stay
    left = sorted(os.listdir(d))
    assert "bs_0_709.ckpt" not in left and "bs_1064_1419.ckpt" in left and "bs_3_17.ckpt" in left
    assert "bs_709_1064.ckpt" in left


def test_partial_tree_with_a_deep_loaded_node(eng, tmp_path):
    """A file deep below the root forces merges at every depth above it."""
    a, b = 0, 5000
    nodes = [(a, b)]
    while nodes[-1][1] - nodes[-1][0] > 40:  # follow the right half down
        lo, hi = nodes[-1]
        nodes.append((lo + (hi - lo) // 2, hi))
    fa, fb = nodes[-1]
    d = str(tmp_path / "deep")
    os.makedirs(d)
    pkg.ckpt_write_bs(os.path.join(d, f"bs_{fa}_{fb}.ckpt"), *oracle.bs(fa, fb))
    vals, rep = eng.bs_checkpointed(a, b, d)
    assert vals == oracle.bs(a, b)
    assert rep["nodes_loaded"] == 1 and rep["merges"] == len(nodes) - 1
    assert rep["subtrees_computed"] == len(nodes) - 1


def test_bs_checkpointed_negative_range_matches_reference(eng, tmp_path):
    d = str(tmp_path / "neg")
    vals, rep = eng.bs_checkpointed(1000, 1419, d)
    assert vals == oracle.bs(1000, 1419)
    assert same_file(os.path.join(d, "bs_1000_1419.ckpt"), os.path.join(CKPT, "bs_1000_1419.ckpt"))
    vals2, rep2 = eng.bs_checkpointed(1000, 1419, d)
    assert vals2 == vals and rep2["root_loaded"] == 1 and rep2["subtrees_computed"] == 0
    for name, (a, b) in (("bs_5_6.ckpt", (5, 6)),):
        d1 = str(tmp_path / "leaf")
        vals, _ = eng.bs_checkpointed(a, b, d1)
        assert vals == oracle.bs(a, b)
        assert same_file(os.path.join(d1, name), os.path.join(CKPT, name))


def test_1_5m_digits_files_match_reference_sha(eng, tmp_path):
    g = json.load(open(os.path.join(GOLDEN, "ckpt_golden.json")))["1500000"]
    d = str(tmp_path / "m15")
    got, rep = eng.pi_checkpointed(1_500_000, d)
    assert hashlib.sha256(got).hexdigest() == g["digits_sha256"]
    assert sha(os.path.join(d, g["bs_file"])) == g["bs_sha256"]
    assert sha(os.path.join(d, g["pi_int_file"])) == g["pi_int_sha256"]
    got2, rep2 = eng.pi_checkpointed(1_500_000, d)
    assert got2 == got and rep2["root_loaded"] == 1 and rep2["pi_int_loaded"] == 1


def test_100m_digits_resume_crosses_staging_chunks(eng, tmp_path):
    """pi_int at 100M digits is 41.5 MB and the root file ~0.3 GB: both stream through more than
    one 32 MB staging buffer in each direction."""
    golden = json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["100000000"]
    d = str(tmp_path / "m100")
    got, rep = eng.pi_checkpointed(100_000_000, d)
    assert hashlib.sha256(got).hexdigest() == golden["sha256"]
    assert rep["root_saved"] == 1 and rep["pi_int_saved"] == 1
    assert os.path.getsize(os.path.join(d, "pi_int_100000000.ckpt")) > 40_000_000
    os.remove(os.path.join(d, "pi_int_100000000.ckpt"))  # resume the splitting only
    got2, rep2 = eng.pi_checkpointed(100_000_000, d)
    assert rep2["root_loaded"] == 1 and rep2["pi_int_saved"] == 1
    assert got2 == got
    got3, rep3 = eng.pi_checkpointed(100_000_000, d)
    assert rep3["root_loaded"] == 1 and rep3["pi_int_loaded"] == 1
    assert got3 == got


def test_cli_checkpoint_flag(tmp_path):
    d = str(tmp_path / "cli")
    out = str(tmp_path / "pi.txt")
    cmd = [pkg.PI_B200_BIN, "--batched", "--digits", "20000", "--checkpoint", d, "--output", out]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    for name in ("bs_0_1419.ckpt", "pi_int_20000.ckpt"):
        assert same_file(os.path.join(d, name), os.path.join(CKPT, name))
    first = open(out, "rb").read()
    assert first.decode() == pi_from_pi_int_file(os.path.join(CKPT, "pi_int_20000.ckpt"))
    subprocess.run(cmd + ["--resume", "--verbose"], check=True, stdout=subprocess.DEVNULL)
    assert open(out, "rb").read() == first
