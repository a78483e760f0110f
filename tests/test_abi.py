"""CPU tests of the C ABI surface: the library loads without a GPU, exports every function
declared in include/*.h, and rejects bad arguments without touching a device."""
import ctypes
import subprocess

import pytest

from helpers import pkg


@pytest.mark.parametrize("header", sorted(pkg.ABI))
def test_library_exports_every_declared_symbol(header):
    import glob
    import os

    assert sorted(glob.glob(os.path.join(pkg.ROOT, "include", "*.h"))) == sorted(pkg.ABI)
    libpath = pkg.ABI[header]
    declared = pkg.declared_symbols(header)
    assert declared
    lib = ctypes.CDLL(libpath)  # loads without a GPU
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(declared) <= exported


def test_version_and_limits():
    lib = pkg.load_library()
    assert lib.pg_version() >= 0x000100
    assert lib.pg_mul_max_limbs() == 1 << 25


def test_create_rejects_bad_device_without_gpu():
    lib = pkg.load_library()
    ctx = ctypes.c_void_p()
    assert lib.pg_create(-1, ctypes.byref(ctx)) == pkg.PG_ERR_BAD_ARG
    assert not ctx.value


def test_null_context_is_rejected():
    lib = pkg.load_library()
    n = ctypes.c_size_t(0)
    assert lib.pg_mul(None, None, 0, None, 0, None, 0, ctypes.byref(n)) == pkg.PG_ERR_BAD_ARG
    assert lib.pg_sync(None) == pkg.PG_ERR_BAD_ARG
    assert lib.pg_last_error(None) == b"null context"


def test_limb_helpers_roundtrip():
    for x in [0, 1, 2**64 - 1, 2**64, 3**5000, 10**300 + 17]:
        assert pkg.limbs_to_int(pkg.int_to_limbs(x)) == x
    a = pkg.random_operand(5, 3)
    assert int(a[-1]) >> 63 == 1
    assert list(pkg.splitmix64(0, 1)) == [0xE220A8397B1DCDAF]


def test_size_checks_do_not_wrap_around():
    # na + nb would wrap around size_t: pg_mul_noalloc must still reject the lengths before it
    # touches memory or the device (these calls return before any CUDA call)
    lib = pkg.load_library()
    big = ctypes.c_size_t(-1).value
    f = lib.pg_mul_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    for na, nb in [(big, 1), (big, 2), (1, big), (big, big), (16384, 1)]:
        assert f(16, na, 16, nb, 16, None) == pkg.PG_ERR_TOO_LARGE, (na, nb)
