"""GPU test of pg_mul_noalloc, the product entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc (another framework owns the allocator, or a
callback where allocating is not allowed); its scratch lives in fixed device arrays inside
the library. The test calls it through the C ABI twice in a row and checks each result
against the existing entry point pg_mul_device, bit for bit (integer products: the
tolerance is zero), and against the oracle. This file sorts last so that a run stopping at
the first failure has run every other test already; it also passes alone in a fresh process
(the first call on the device does the set-up). Shapes cover the one-pass plans (na + nb <= 4096
limbs), the two-pass plans and an empty operand.
"""
import ctypes

import numpy as np
import pytest

from helpers import oracle, pkg

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    lib = pkg.load_library()
    f = lib.pg_mul_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return lib, f


def test_noalloc_matches_existing_entry_point_twice():
    import torch

    lib, noalloc = _noalloc_fn()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    eng = pkg.Engine(0)
    try:
        # calls in a row, different shapes: two-pass plans (L = 2^14, and 2^15 at the largest size
        # accepted), one-pass plans (na + nb <= 4096: L = 2^6, 2^9, 2^13) and an empty operand
        for na, nb, seed in [(5000, 3001, 1), (8192, 8192, 2), (1, 1, 3), (100, 37, 4), (3000, 1096, 5),
                             (0, 5, 6), (4096, 4096, 7)]:
            a = pkg.random_operand(na, seed)
            b = pkg.random_operand(nb, seed + 100)
            # an empty operand still gets a valid (16-byte aligned) device address
            da = torch.from_numpy(a.view(np.int64)).cuda() if na else torch.zeros(2, dtype=torch.int64, device="cuda")
            db = torch.from_numpy(b.view(np.int64)).cuda() if nb else torch.zeros(2, dtype=torch.int64, device="cuda")
            out_new = torch.full((na + nb,), -1, dtype=torch.int64, device="cuda")
            out_ref = torch.zeros(na + nb, dtype=torch.int64, device="cuda")
            torch.cuda.synchronize()
            st = noalloc(da.data_ptr(), na, db.data_ptr(), nb, out_new.data_ptr(), stream)
            assert st == pkg.PG_OK, st
            assert lib.pg_mul_device(eng.ctx, da.data_ptr(), na, db.data_ptr(), nb, out_ref.data_ptr()) == 0
            assert lib.pg_sync(eng.ctx) == 0
            got = out_new.cpu().numpy().view(np.uint64)
            ref = out_ref.cpu().numpy().view(np.uint64)
            assert np.array_equal(got, ref)
            exp = oracle.mul_gmp(a, b) if na and nb else np.zeros(0, dtype=np.uint64)
            assert np.array_equal(got[: len(exp)], exp) and not got[len(exp):].any()
        # beyond the stated maximum: rejected with a clear status, nothing touched
        assert noalloc(da.data_ptr(), 8192, db.data_ptr(), 8193, out_new.data_ptr(), stream) == pkg.PG_ERR_TOO_LARGE
    finally:
        eng.close()
