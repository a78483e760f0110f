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


def test_captured_level_replays_over_new_operands(eng):
    # One level of products (mul, square, a*b + c*d, a*b - c*d, an empty product) captured once
    # (pg_graph_capture_level), replayed twice over new operand contents in the same buffers, with
    # an unrelated batch on the context in between; every replay equals the oracle.
    import ctypes

    lib = eng.lib
    shapes = [(700, 300), (2048, None), (500, 400, 450, 420, 1), (900, 800, 600, 500, -1), (0, 64)]
    bufs, jobs, outs = [], [], []

    def operand(n, seed, big=False):
        x = pkg.random_operand(n, seed)
        if big and n:
            x[-1] |= np.uint64(1 << 63)
        return x

    for i, sh in enumerate(shapes):
        na, nb = sh[0], sh[1]
        acc = sh[4] if len(sh) > 2 else 0
        nc, nd = (sh[2], sh[3]) if acc else (0, 0)
        ba = eng.buffer(operand(na, 10 + i)) if na else eng.buffer(np.zeros(2, dtype=np.uint64))
        bb = eng.buffer(operand(nb, 20 + i)) if nb else None
        bc = eng.buffer(operand(nc, 30 + i)) if acc else None
        bd = eng.buffer(operand(nd, 40 + i)) if acc else None
        top = max(na + (nb if nb is not None else na), nc + nd) + (1 if acc > 0 else 0)
        bo = pkg.DeviceBuffer(eng, max(top, 1), None)
        bufs.append((ba, bb, bc, bd, bo, top, na, nb, nc, nd, acc))
        jobs.append(pkg.PgJob(ba.ptr, na, bb.ptr if bb else None, nb or 0, bc.ptr if bc else None, nc,
                              bd.ptr if bd else None, nd, acc, bo.ptr, bo.cap))
    arr = (pkg.PgJob * len(jobs))(*jobs)
    g = ctypes.c_void_p()
    assert lib.pg_graph_capture_level(eng.ctx, arr, len(jobs), ctypes.byref(g)) == pkg.PG_OK
    try:
        for rep in range(2):
            exp = []
            for i, (ba, bb, bc, bd, bo, top, na, nb, nc, nd, acc) in enumerate(bufs):
                # new contents of the same lengths (for acc = -1, a*b stays larger than c*d)
                seed = 1000 * (rep + 1) + i
                A = operand(na, seed, big=True)
                if na:
                    assert lib.pg_buf_upload(eng.ctx, ba.h, A.ctypes.data_as(pkg._u64p), na) == 0
                a = pkg.limbs_to_int(A)
                b = a
                if nb:
                    B = operand(nb, seed + 1, big=True)
                    assert lib.pg_buf_upload(eng.ctx, bb.h, B.ctypes.data_as(pkg._u64p), nb) == 0
                    b = pkg.limbs_to_int(B)
                v = gmp(a, b) if na else 0
                if acc:
                    C, D = operand(nc, seed + 2), operand(nd, seed + 3)
                    assert lib.pg_buf_upload(eng.ctx, bc.h, C.ctypes.data_as(pkg._u64p), nc) == 0
                    assert lib.pg_buf_upload(eng.ctx, bd.h, D.ctypes.data_as(pkg._u64p), nd) == 0
                    v += acc * gmp(pkg.limbs_to_int(C), pkg.limbs_to_int(D))
                exp.append(v)
            # an unrelated batch between replays
            x, y = rnd(3000, 5 + rep), rnd(2000, 6 + rep)
            assert eng.mul_batch([(x, y)]) == [gmp(x, y)]
            assert lib.pg_graph_launch(g) == pkg.PG_OK
            for (ba, bb, bc, bd, bo, top, *_), v in zip(bufs, exp):
                bo.set_len(top)
                assert pkg.limbs_to_int(bo.download()) == v
    finally:
        lib.pg_graph_destroy(g)
        for t in bufs:
            for x in t[:5]:
                if x is not None:
                    x.free()
