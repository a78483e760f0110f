"""GPU tests of the pass-split autotuner (pg_tune, pg_tune_save, pg_tune_load).

A tuned context must produce products identical to the oracle (libgmp's mpz_mul) at every
transform length it tuned; files with invalid splits are rejected.
"""
import os

import numpy as np
import pytest

from helpers import oracle, pkg

pytestmark = pytest.mark.gpu


def test_tune_save_load_and_products(tmp_path, monkeypatch):
    monkeypatch.setenv("PG_TUNE_FILE", "")  # a context with the built-in splits only
    path = str(tmp_path / "splits.txt")
    with pkg.Engine(0) as eng:
        times = eng.tune(10, 21)
        assert len(times) == 12 and all(t > 0 for t in times)
        eng.tune_save(path)
    lines = [l.split() for l in open(path) if not l.startswith("#")]
    narrow = [l for l in lines if len(l) == 5]
    wide = [l for l in lines if len(l) == 6]
    assert all(l[5] == "64" for l in wide)
    assert [int(l[0]) for l in narrow] == list(range(10, 22))
    assert [int(l[0]) for l in wide] == list(range(9, 21))  # the same products, half the transform length
    for l in narrow + wide:
        logl, npass, *n = map(int, l[:5])
        assert sum(n[:npass]) == logl
    assert all(l[0] == "wide_min_limbs" for l in lines if len(l) == 2)
    with pkg.Engine(0) as eng:
        eng.tune_load(path)
        for wmin in ("1", "0"):  # every product wide, then none
            monkeypatch.setenv("PG_WIDE_MIN_LIMBS", wmin)
            for logl in range(10, 22):
                n = 1 << (logl - 2)
                for na, nb in ((n, n), (n + n // 2 - 3, n // 2 + 1)):
                    a, b = pkg.random_operand(na, 7 * logl), pkg.random_operand(nb, 11 * logl)
                    assert np.array_equal(eng.mul_limbs(a, b), oracle.mul_gmp(a, b)), (wmin, logl, na, nb)


def test_tuned_table_loaded_at_context_creation(tmp_path, monkeypatch):
    """PG_TUNE_FILE (or tune_b200.txt beside the library) is applied when the context is made."""
    src = str(tmp_path / "mine.txt")
    open(src, "w").write("# test\n14 2 7 7 0\n20 2 10 10 0\n24 3 5 6 13\n")
    monkeypatch.setenv("PG_TUNE_FILE", src)
    out = str(tmp_path / "saved.txt")
    with pkg.Engine(0) as eng:
        eng.tune_save(out)
        for n in (1 << 12, 1 << 18, 1 << 22):
            a, b = pkg.random_operand(n, 5), pkg.random_operand(n - 7, 6)
            assert np.array_equal(eng.mul_limbs(a, b), oracle.mul_gmp(a, b))
    saved = [l.split() for l in open(out) if not l.startswith("#")]
    assert saved == [["14", "2", "7", "7", "0"], ["20", "2", "10", "10", "0"], ["24", "3", "5", "6", "13"]]


@pytest.mark.parametrize("text", ["14 2 7 8 0\n", "20 2 4 16 0\n", "26 1 26 0 0\n", "x\n", "14 4 5 5 4\n",
                                  "26 3 6 8 12 64\n", "14 2 7 7 0 48\n"])
def test_tune_load_rejects_invalid(tmp_path, text, monkeypatch):
    path = str(tmp_path / "bad.txt")
    open(path, "w").write(text)
    with pkg.Engine(0) as eng:
        with pytest.raises(pkg.PgError) as ei:
            eng.tune_load(path)
        assert ei.value.status == pkg.PG_ERR_BAD_ARG
        a, b = pkg.random_operand(5000, 1), pkg.random_operand(4000, 2)
        assert np.array_equal(eng.mul_limbs(a, b), oracle.mul_gmp(a, b))
