"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke() and bench.py's CPU
baseline may use it; the product never does).

ctypes bindings of
  oracle/_build/liboracle.so  CPU restatement of the reference's hot-path arithmetic (oracle.h)
  oracle/_ref/libpiref.so     the reference's own CPU sources compiled unchanged + ref_shim.cpp
  oracle/_ref/pi_compute_ref  the reference's own CLI program
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBORACLE = os.path.join(HERE, "_build", "liboracle.so")
LIBPIREF = os.path.join(HERE, "_ref", "libpiref.so")
PI_COMPUTE_REF = os.path.join(HERE, "_ref", "pi_compute_ref")

_u64p = ctypes.POINTER(ctypes.c_uint64)
_o = None
_r = None


def build() -> None:
    """Compile the restatement library, and the reference build when its sources are mounted."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _o
    if _o is None:
        if not os.path.exists(LIBORACLE):
            build()
        o = ctypes.CDLL(LIBORACLE)
        for name in ("oracle_mul_schoolbook", "oracle_mul_karatsuba", "oracle_mul_gmp"):
            f = getattr(o, name)
            f.argtypes = [_u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, _u64p]
            f.restype = None
        o.oracle_int_new.restype = ctypes.c_void_p
        o.oracle_int_free.argtypes = [ctypes.c_void_p]
        o.oracle_int_sign.argtypes = [ctypes.c_void_p]
        o.oracle_int_sign.restype = ctypes.c_int
        o.oracle_int_size.argtypes = [ctypes.c_void_p]
        o.oracle_int_size.restype = ctypes.c_size_t
        o.oracle_int_get_limbs.argtypes = [ctypes.c_void_p, _u64p]
        o.oracle_int_set_limbs.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_size_t, ctypes.c_int]
        o.oracle_bs.argtypes = [ctypes.c_ulong, ctypes.c_ulong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        o.oracle_bs_merge.argtypes = [ctypes.c_void_p] * 9
        o.oracle_terms_needed.argtypes = [ctypes.c_size_t]
        o.oracle_terms_needed.restype = ctypes.c_ulong
        _o = o
    return _o


def _mul(fn, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.zeros(len(a) + len(b), dtype=np.uint64)
    fn(a.ctypes.data_as(_u64p), len(a), b.ctypes.data_as(_u64p), len(b), out.ctypes.data_as(_u64p))
    n = len(out)
    while n and out[n - 1] == 0:
        n -= 1
    return out[:n]


def mul_gmp(a, b):
    return _mul(lib().oracle_mul_gmp, a, b)


def mul_schoolbook(a, b):
    return _mul(lib().oracle_mul_schoolbook, a, b)


def mul_karatsuba(a, b):
    return _mul(lib().oracle_mul_karatsuba, a, b)


class OInt:
    def __init__(self):
        self.h = lib().oracle_int_new()

    def __del__(self):
        try:
            lib().oracle_int_free(self.h)
        except Exception:
            pass

    def value(self) -> int:
        o = lib()
        n = o.oracle_int_size(self.h)
        buf = np.zeros(max(n, 1), dtype=np.uint64)
        o.oracle_int_get_limbs(self.h, buf.ctypes.data_as(_u64p))
        v = int.from_bytes(buf[:n].astype("<u8").tobytes(), "little")
        return -v if o.oracle_int_sign(self.h) < 0 else v


def bs(a: int, b: int) -> tuple[int, int, int]:
    """Oracle P(a,b), Q(a,b), R(a,b) (restatement over libgmp)."""
    P, Q, R = OInt(), OInt(), OInt()
    lib().oracle_bs(a, b, P.h, Q.h, R.h)
    return P.value(), Q.value(), R.value()


def terms_needed(digits: int) -> int:
    return int(lib().oracle_terms_needed(digits))


# ------------------------------------------------------------------ the reference build
def ref_available() -> bool:
    return os.path.exists(LIBPIREF) and os.path.exists(PI_COMPUTE_REF)


def ref() -> ctypes.CDLL:
    global _r
    if _r is None:
        r = ctypes.CDLL(LIBPIREF)
        cp = ctypes.POINTER(ctypes.c_char_p)
        r.ref_bs.argtypes = [ctypes.c_ulong, ctypes.c_ulong, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p,
                             ctypes.c_void_p]
        r.ref_bs.restype = ctypes.c_int
        r.ref_bs_checkpoint.argtypes = [ctypes.c_ulong, ctypes.c_ulong, ctypes.c_uint, ctypes.c_char_p]
        r.ref_bs_checkpoint.restype = ctypes.c_int
        r.ref_pi.argtypes = [ctypes.c_ulong, ctypes.c_uint]
        r.ref_pi.restype = ctypes.c_void_p
        r.ref_terms_needed.argtypes = [ctypes.c_ulong]
        r.ref_terms_needed.restype = ctypes.c_ulong
        r.ref_free.argtypes = [ctypes.c_void_p]
        r.ref_gmp_mul.argtypes = [_u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, _u64p]
        r.ref_gmp_mul.restype = None
        _r = r
    return _r


def ref_bs(a: int, b: int, threads: int = 1) -> tuple[int, int, int]:
    """P/Q/R from the reference's own BinarySplitting::compute with GmpMultiplier."""
    r = ref()
    ps = [ctypes.c_void_p() for _ in range(3)]
    st = r.ref_bs(a, b, threads, *(ctypes.byref(p) for p in ps))
    if st != 0:
        raise RuntimeError("ref_bs failed")
    out = []
    for p in ps:
        s = ctypes.cast(p, ctypes.c_char_p).value.decode()
        r.ref_free(p)
        out.append(int(s, 16))
    return tuple(out)


def ref_bs_checkpoint(a: int, b: int, directory: str, threads: int = 1) -> str:
    """Path of bs_<a>_<b>.ckpt as the reference's own BinarySplitting writes it into `directory`."""
    if ref().ref_bs_checkpoint(a, b, threads, directory.encode()) != 0:
        raise RuntimeError("ref_bs_checkpoint failed")
    return os.path.join(directory, f"bs_{a}_{b}.ckpt")


def ref_pi(digits: int, threads: int = 1) -> str:
    """The reference PiEngine's digit string "3.xxxx" for `digits` digits."""
    r = ref()
    p = r.ref_pi(digits, threads)
    if not p:
        raise RuntimeError("ref_pi failed")
    s = ctypes.cast(p, ctypes.c_char_p).value.decode()
    r.ref_free(p)
    return s


def ref_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Product through the reference's own GmpMultiplier::multiply (compiled from its sources)."""
    return _mul(ref().ref_gmp_mul, a, b)


# ------------------------------------------------------------------ the reference with the drop-in
LIBPIREF_B200 = os.path.join(HERE, "_ref", "libpiref_b200.so")
_rb = None


def refb() -> ctypes.CDLL:
    """oracle/_ref/libpiref_b200.so: the reference's own BinarySplitting and PiEngine, compiled
    unchanged, with the library's pi::B200Multiplier behind their Multiplier& (needs a GPU to run)."""
    global _rb
    if _rb is None:
        r = ctypes.CDLL(LIBPIREF_B200)
        r.refb_bs.argtypes = [ctypes.c_ulong, ctypes.c_ulong, ctypes.c_uint, ctypes.c_size_t, ctypes.c_int,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong)]
        r.refb_bs.restype = ctypes.c_int
        r.refb_pi.argtypes = [ctypes.c_ulong, ctypes.c_uint, ctypes.c_size_t, ctypes.c_int,
                              ctypes.POINTER(ctypes.c_ulonglong)]
        r.refb_pi.restype = ctypes.c_void_p
        r.refb_free.argtypes = [ctypes.c_void_p]
        _rb = r
    return _rb


def refb_bs(a: int, b: int, threshold: int, threads: int = 1, device: int = 0):
    """(P, Q, R, products on the B200) from the reference's BinarySplitting::compute over B200Multiplier."""
    r = refb()
    ps = [ctypes.c_void_p() for _ in range(3)]
    calls = ctypes.c_ulonglong(0)
    if r.refb_bs(a, b, threads, threshold, device, *(ctypes.byref(p) for p in ps), ctypes.byref(calls)) != 0:
        raise RuntimeError("refb_bs failed")
    out = []
    for p in ps:
        out.append(int(ctypes.cast(p, ctypes.c_char_p).value.decode(), 16))
        r.refb_free(p)
    return out[0], out[1], out[2], calls.value


def refb_pi(digits: int, threshold: int, threads: int = 1, device: int = 0):
    """("3." + digits, products on the B200) from the reference's PiEngine over B200Multiplier."""
    r = refb()
    calls = ctypes.c_ulonglong(0)
    p = r.refb_pi(digits, threads, threshold, device, ctypes.byref(calls))
    if not p:
        raise RuntimeError("refb_pi failed")
    s = ctypes.cast(p, ctypes.c_char_p).value.decode()
    r.refb_free(p)
    return s, calls.value
