"""GPU parity tests of pg_mul_batch and the pg_buf device buffers (C ABI of libpigpu.so).

A batch replaces a tree level's sequence of Multiplier calls (the reference issues the
products of each merge one at a time, binary_splitting.cpp:183-238, and adds R with mpz_add,
:199-200). Every result is compared bit-exactly with the oracle (libgmp's mpz_mul) and plain
integer addition/subtraction of oracle products.
"""
import numpy as np
import pytest

from helpers import oracle, pkg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = pkg.Engine(0)
    yield e
    e.close()


def gmp(a: int, b: int) -> int:
    return pkg.limbs_to_int(oracle.mul_gmp(pkg.int_to_limbs(a), pkg.int_to_limbs(b)))


def rnd(n: int, seed: int) -> int:
    return pkg.limbs_to_int(pkg.random_operand(n, seed)) if n else 0


def test_buffer_round_trip(eng):
    a = pkg.random_operand(1000, 7)
    b = eng.buffer(a)
    assert b.len == 1000
    assert np.array_equal(b.download(), a)
    b.free()


def test_mixed_batch_matches_oracle(eng):
    rng = np.random.default_rng(11)
    jobs, exp = [], []
    for i in range(120):
        kind = i % 4
        na = int(rng.integers(1, 3000))
        nb = int(rng.integers(1, 3000))
        a, b = rnd(na, 100 + i), rnd(nb, 500 + i)
        if kind == 0:
            jobs.append((a, b)); exp.append(gmp(a, b))
        elif kind == 1:
            jobs.append((a, None)); exp.append(gmp(a, a))
        elif kind == 2:
            c, d = rnd(int(rng.integers(1, 3000)), 900 + i), rnd(int(rng.integers(1, 3000)), 1300 + i)
            jobs.append((a, b, c, d, 1)); exp.append(gmp(a, b) + gmp(c, d))
        else:
            c = rnd(max(1, na // 3), 1700 + i)
            d = rnd(max(1, nb // 3), 2100 + i)
            jobs.append((a, b, c, d, -1)); exp.append(gmp(a, b) - gmp(c, d))
    got = eng.mul_batch(jobs)
    for i, (g, e) in enumerate(zip(got, exp)):
        assert g == e, i


def test_synthetic_log_uniform_batch(eng):
    """Products with sizes drawn log-uniform in [2^6, 2^16] limbs from one seed (the shape of the
    synthetic batch workload, reduced in count and top size for the oracle)."""
    rng = np.random.default_rng(2024)
    n = 256
    la = rng.uniform(6, 16, n)
    lb = rng.uniform(6, 16, n)
    jobs, exp = [], []
    for i in range(n):
        a, b = rnd(int(2 ** la[i]), 10_000 + i), rnd(int(2 ** lb[i]), 20_000 + i)
        jobs.append((a, b))
        exp.append(gmp(a, b))
    got = eng.mul_batch(jobs)
    assert got == exp


def test_accumulate_like_bs_merge(eng):
    """R = Qr*Rl + Pl*Rr (and the subtracting form) at sizes where the transform is multi-pass."""
    for n in (5000, 70000):
        qr, rl, pl, rr = (rnd(n, s) for s in (1, 2, 3, 4))
        got = eng.mul_batch([(qr, rl, pl, rr, 1), (qr, rl, pl >> 64, rr, -1), (qr, None, rl, None, 1)])
        assert got[0] == gmp(qr, rl) + gmp(pl, rr)
        assert got[1] == gmp(qr, rl) - gmp(pl >> 64, rr)
        assert got[2] == gmp(qr, qr) + gmp(rl, rl)


def test_empty_operands_and_carry_stress(eng):
    ones = (1 << (64 * 2048)) - 1
    got = eng.mul_batch([(0, 5), (ones, ones), (ones, None), (7, 0, 0, 9, 1), (ones, ones, ones, 1, -1)])
    assert got == [0, ones * ones, ones * ones, 0, ones * ones - ones]


def test_batch_errors(eng):
    with pytest.raises(pkg.PgError) as ei:
        eng.mul_batch([(rnd(10, 1), rnd(10, 2), rnd(40, 3), rnd(40, 4), -1)])  # negative result
    assert ei.value.status == pkg.PG_ERR_BAD_ARG
    # the context stays usable after the error
    a, b = rnd(300, 5), rnd(200, 6)
    assert eng.mul_batch([(a, b)]) == [gmp(a, b)]
