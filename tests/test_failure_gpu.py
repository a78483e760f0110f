"""GPU tests of the failure paths: a bounded device wait that runs out, and a device allocation
that fails. Both failures are made on the host, without faulting, trapping or hanging the GPU:

* the carry look-back wait (crt_carry_kernel) gets a short poll limit, and one block is kept
  from publishing its carry (PG_TEST_CRT_SPIN_LIMIT / PG_TEST_CRT_WITHHOLD, read by the library
  at every launch), so that the next block's wait runs out: the product must report
  PG_ERR_TIMEOUT, and the same context must then compute the product correctly;
* the look-back wait of the one-launch long sums (add_onepass_kernel) the same way
  (PG_TEST_ADD_SPIN_LIMIT / PG_TEST_ADD_WITHHOLD): a reciprocal whose sums span many segments must
  report PG_ERR_TIMEOUT, and then be exact;
* every library device allocation fails while PG_TEST_FAIL_DEVICE_ALLOC is set: a product that
  needs a larger workspace, and a device buffer, must report PG_ERR_OOM, and the context must
  work once the variable is cleared.

The reference's only failure path is the C++ exception its CUDA_CHECK throws
(src/gpu/int_ntt.cu:20-26); here failures are status codes and the context stays usable.
"""
import ctypes
import os

import numpy as np
import pytest

from helpers import oracle, pkg

pytestmark = pytest.mark.gpu


@pytest.fixture
def eng():
    e = pkg.Engine(0)
    yield e
    e.close()


def _with_env(env, fn):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return fn()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def test_lookback_wait_runs_out_and_context_recovers(eng):
    # 2^15 x 2^15 limbs in the 32-bit configuration (the one whose CRT carries look back):
    # 2^17 output words, 32 carry blocks; block 2 never publishes its carry
    a = pkg.random_operand(1 << 15, 11)
    b = pkg.random_operand(1 << 15, 12)
    narrow = {"PG_WIDE_MIN_LIMBS": "0"}
    with pytest.raises(pkg.PgError) as err:
        _with_env(dict(narrow, PG_TEST_CRT_SPIN_LIMIT="2000", PG_TEST_CRT_WITHHOLD="2"), lambda: eng.mul_limbs(a, b))
    assert err.value.status == pkg.PG_ERR_TIMEOUT
    assert "look-back" in eng.last_error()
    exp = oracle.mul_gmp(a, b)
    assert np.array_equal(_with_env(narrow, lambda: eng.mul_limbs(a, b)), exp)
    assert np.array_equal(eng.mul_limbs(a, b), exp)


def test_sum_lookback_wait_runs_out_and_context_recovers(eng):
    # a 2^21-bit reciprocal: its top Newton level sums numbers of 2^15 - 2^16 limbs (16-32
    # segments of 2048); segment 2 never publishes its status, so the later segments' waits run out
    k = 1 << 21
    r = pkg.limbs_to_int(pkg.random_operand(k // 64, 21)) | (1 << (k - 1))
    with pytest.raises(pkg.PgError) as err:
        _with_env({"PG_TEST_ADD_SPIN_LIMIT": "2000", "PG_TEST_ADD_WITHHOLD": "2"}, lambda: eng.recip_floor(r))
    assert err.value.status == pkg.PG_ERR_TIMEOUT
    assert "sum look-back" in eng.last_error()
    assert eng.recip_floor(r) == (1 << (2 * k)) // r


def test_device_allocation_failure_is_oom_and_context_recovers(eng):
    small = pkg.random_operand(64, 1)
    assert np.array_equal(eng.mul_limbs(small, small), oracle.mul_gmp(small, small))
    a = pkg.random_operand(1 << 18, 21)  # needs a larger residue workspace than the first product
    b = pkg.random_operand(1 << 17, 22)
    with pytest.raises(pkg.PgError) as err:
        _with_env({"PG_TEST_FAIL_DEVICE_ALLOC": "1"}, lambda: eng.mul_limbs(a, b))
    assert err.value.status == pkg.PG_ERR_OOM
    buf = ctypes.c_void_p()
    st = _with_env({"PG_TEST_FAIL_DEVICE_ALLOC": "1"},
                   lambda: eng.lib.pg_buf_alloc(eng.ctx, 1 << 20, ctypes.byref(buf)))
    assert st == pkg.PG_ERR_OOM and not buf.value
    assert np.array_equal(eng.mul_limbs(a, b), oracle.mul_gmp(a, b))
    assert eng.lib.pg_buf_alloc(eng.ctx, 1 << 20, ctypes.byref(buf)) == pkg.PG_OK and buf.value
    eng.lib.pg_buf_free(eng.ctx, buf)


def test_pi_allocation_failure_is_oom_and_context_recovers():
    """A fresh context computing pi with every device allocation failing: the splitting and the
    helper thread (sqrt(10005) and the powers of ten on the second stream) both fail; the call must
    report PG_ERR_OOM after the helper has finished, and the same context must then compute the
    digits."""
    e = pkg.Engine(0)
    try:
        with pytest.raises(pkg.PgError) as err:
            _with_env({"PG_TEST_FAIL_DEVICE_ALLOC": "1"}, lambda: e.pi(200_000))
        assert err.value.status == pkg.PG_ERR_OOM
        ref = open(os.path.join(os.path.dirname(__file__), "golden", "pi_1000.txt")).read().strip()
        assert e.pi(200_000).decode()[:1002] == ref
    finally:
        e.close()
