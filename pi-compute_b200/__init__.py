"""pi-compute_b200: exact big-integer products on one B200 behind the pi::Multiplier boundary.

Python side of the package: a ctypes binding of the C ABI in include/pi_b200.h
(libpigpu.so) used by tests, smoke checks and the benchmark, plus operand
helpers. The product path is native; nothing here computes a product on the CPU.
If the shared library is missing the import of :class:`Engine` fails loudly.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIBPIGPU = os.path.join(HERE, "libpigpu.so")
LIBPIB200 = os.path.join(HERE, "libpib200.so")
PI_B200_BIN = os.path.join(HERE, "pi_b200")
HEADERS = [os.path.join(ROOT, "include", "pi_b200.h")]
# header -> library that must export every function it declares
ABI = {os.path.join(ROOT, "include", "pi_b200.h"): LIBPIGPU,
       os.path.join(ROOT, "include", "pi_b200_engine.h"): LIBPIB200}

PG_OK = 0
PG_ERR_OOM = 1
PG_ERR_TOO_LARGE = 2
PG_ERR_BAD_ARG = 3
PG_ERR_DEVICE = 4
PG_ERR_TIMEOUT = 5
PG_ERR_INTERNAL = 6
PG_ERR_IO = 7

_u64p = ctypes.POINTER(ctypes.c_uint64)
_sizep = ctypes.POINTER(ctypes.c_size_t)


class PgError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"pg status {status}: {msg}")
        self.status = status


_lib: Optional[ctypes.CDLL] = None


class PgJob(ctypes.Structure):
    """struct pg_job of include/pi_b200.h (device addresses and limb counts)."""
    _fields_ = [("a", ctypes.c_void_p), ("na", ctypes.c_size_t), ("b", ctypes.c_void_p), ("nb", ctypes.c_size_t),
                ("c", ctypes.c_void_p), ("nc", ctypes.c_size_t), ("d", ctypes.c_void_p), ("nd", ctypes.c_size_t),
                ("acc", ctypes.c_int), ("out", ctypes.c_void_p), ("out_cap", ctypes.c_size_t)]


class PgCkptReport(ctypes.Structure):
    """struct pg_ckpt_report of include/pi_b200.h."""
    _fields_ = [("root_loaded", ctypes.c_int), ("root_saved", ctypes.c_int), ("pi_int_loaded", ctypes.c_int),
                ("pi_int_saved", ctypes.c_int), ("nodes_loaded", ctypes.c_size_t),
                ("subtrees_computed", ctypes.c_size_t), ("merges", ctypes.c_size_t)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def load_library(path: str = LIBPIGPU) -> ctypes.CDLL:
    """Load libpigpu.so and declare the C ABI signatures. Raises if the library is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} not built: run `python pi-compute_b200/build.py`")
    lib = ctypes.CDLL(path)
    lib.pg_version.restype = ctypes.c_int
    lib.pg_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    lib.pg_create.restype = ctypes.c_int
    lib.pg_destroy.argtypes = [ctypes.c_void_p]
    lib.pg_destroy.restype = None
    lib.pg_last_error.argtypes = [ctypes.c_void_p]
    lib.pg_last_error.restype = ctypes.c_char_p
    lib.pg_mul_max_limbs.restype = ctypes.c_size_t
    lib.pg_mul.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, _u64p,
                           ctypes.c_size_t, _sizep]
    lib.pg_mul.restype = ctypes.c_int
    lib.pg_sqr.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, _sizep]
    lib.pg_sqr.restype = ctypes.c_int
    lib.pg_mul_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                  ctypes.c_size_t, ctypes.c_void_p]
    lib.pg_mul_device.restype = ctypes.c_int
    lib.pg_sqr_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.pg_sqr_device.restype = ctypes.c_int
    lib.pg_sync.argtypes = [ctypes.c_void_p]
    lib.pg_sync.restype = ctypes.c_int
    lib.pg_stream.argtypes = [ctypes.c_void_p]
    lib.pg_stream.restype = ctypes.c_void_p
    lib.pg_launch_count.argtypes = [ctypes.c_void_p]
    lib.pg_launch_count.restype = ctypes.c_uint64
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    lib.pg_buf_alloc.argtypes = [vp, sz, ctypes.POINTER(vp)]
    lib.pg_buf_alloc.restype = ctypes.c_int
    lib.pg_buf_free.argtypes = [vp, vp]
    lib.pg_buf_free.restype = None
    lib.pg_buf_upload.argtypes = [vp, vp, _u64p, sz]
    lib.pg_buf_upload.restype = ctypes.c_int
    lib.pg_buf_download.argtypes = [vp, vp, _u64p, sz, _sizep]
    lib.pg_buf_download.restype = ctypes.c_int
    lib.pg_buf_device.argtypes = [vp]
    lib.pg_buf_device.restype = vp
    lib.pg_buf_len.argtypes = [vp]
    lib.pg_buf_len.restype = sz
    lib.pg_buf_capacity.argtypes = [vp]
    lib.pg_buf_capacity.restype = sz
    lib.pg_buf_set_len.argtypes = [vp, sz]
    lib.pg_buf_set_len.restype = ctypes.c_int
    lib.pg_mul_batch.argtypes = [vp, ctypes.POINTER(PgJob), sz]
    lib.pg_mul_batch.restype = ctypes.c_int
    lib.pg_graph_capture_level.argtypes = [vp, ctypes.POINTER(PgJob), sz, ctypes.POINTER(vp)]
    lib.pg_graph_capture_level.restype = ctypes.c_int
    lib.pg_graph_launch.argtypes = [vp]
    lib.pg_graph_launch.restype = ctypes.c_int
    lib.pg_graph_destroy.argtypes = [vp]
    lib.pg_graph_destroy.restype = None
    lib.pg_recip_floor.argtypes = [vp, _u64p, sz, _u64p, sz, _sizep]
    lib.pg_recip_floor.restype = ctypes.c_int
    lib.pg_mul_wrap.argtypes = [vp, _u64p, sz, _u64p, sz, ctypes.c_int, _u64p, sz, _sizep]
    lib.pg_mul_wrap.restype = ctypes.c_int
    lib.pg_sqrt_scaled.argtypes = [vp, ctypes.c_uint64, sz, _u64p, sz, _sizep]
    lib.pg_sqrt_scaled.restype = ctypes.c_int
    lib.pg_to_decimal.argtypes = [vp, _u64p, sz, sz, ctypes.c_char_p]
    lib.pg_to_decimal.restype = ctypes.c_int
    lib.pg_pi_finish.argtypes = [vp, _u64p, sz, _u64p, sz, sz, ctypes.c_char_p]
    lib.pg_pi_finish.restype = ctypes.c_int
    lib.pg_pi.argtypes = [vp, sz, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
    lib.pg_pi.restype = ctypes.c_int
    lib.pg_tune.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.pg_tune.restype = ctypes.c_int
    lib.pg_tune_save.argtypes = [vp, ctypes.c_char_p]
    lib.pg_tune_save.restype = ctypes.c_int
    lib.pg_tune_load.argtypes = [vp, ctypes.c_char_p]
    lib.pg_tune_load.restype = ctypes.c_int
    lib.pg_bs.argtypes = [vp, ctypes.c_ulong, ctypes.c_ulong, ctypes.c_void_p, _u64p, _u64p, sz, _sizep,
                          ctypes.POINTER(ctypes.c_int)]
    lib.pg_bs.restype = ctypes.c_int
    p3 = ctypes.c_void_p * 3
    lib.pg_ckpt_write_bs.argtypes = [ctypes.c_char_p, p3, ctypes.c_size_t * 3, ctypes.c_int * 3]
    lib.pg_ckpt_write_bs.restype = ctypes.c_int
    lib.pg_ckpt_read_bs.argtypes = [ctypes.c_char_p, ctypes.c_void_p, sz, ctypes.c_size_t * 3, ctypes.c_int * 3]
    lib.pg_ckpt_read_bs.restype = ctypes.c_int
    lib.pg_ckpt_write_pi_int.argtypes = [ctypes.c_char_p, _u64p, sz]
    lib.pg_ckpt_write_pi_int.restype = ctypes.c_int
    lib.pg_ckpt_read_pi_int.argtypes = [ctypes.c_char_p, ctypes.c_void_p, sz, _sizep]
    lib.pg_ckpt_read_pi_int.restype = ctypes.c_int
    lib.pg_bs_checkpointed.argtypes = [vp, ctypes.c_ulong, ctypes.c_ulong, ctypes.c_char_p, ctypes.c_void_p, _u64p, _u64p,
                                       sz, ctypes.c_size_t * 3, ctypes.c_int * 3, ctypes.POINTER(PgCkptReport)]
    lib.pg_bs_checkpointed.restype = ctypes.c_int
    lib.pg_pi_checkpointed.argtypes = [vp, sz, ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(PgCkptReport)]
    lib.pg_pi_checkpointed.restype = ctypes.c_int
    _lib = lib
    return lib


def declared_symbols(header: str = HEADERS[0]) -> list[str]:
    """Every function name declared in one of include/*.h (the C ABI its library must export)."""
    import re

    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = [m.group(1) for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b((?:pg|pib)_\w+)\s*\(", text,
                                             flags=re.M)]
    return sorted(set(names))


# ------------------------------------------------------------------ limb helpers
def int_to_limbs(x: int) -> np.ndarray:
    """Magnitude of x as little-endian uint64 limbs (empty for 0)."""
    x = abs(int(x))
    n = (x.bit_length() + 63) // 64
    if n == 0:
        return np.zeros(0, dtype=np.uint64)
    return np.frombuffer(x.to_bytes(8 * n, "little"), dtype="<u8").astype(np.uint64)


def limbs_to_int(a: np.ndarray) -> int:
    a = np.ascontiguousarray(a, dtype="<u8")
    return int.from_bytes(a.tobytes(), "little")


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n outputs of the splitmix64 generator started at `seed` (vectorised)."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def random_operand(n: int, seed: int) -> np.ndarray:
    """Uniform random n-limb operand with the top limb's most significant bit set (exact length)."""
    a = splitmix64(seed, n)
    if n:
        a[-1] |= np.uint64(1 << 63)
    return a


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_u64p)


class Engine:
    """One pg_ctx (device context, twiddle tables, workspace) on a CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        ctx = ctypes.c_void_p()
        st = self.lib.pg_create(device, ctypes.byref(ctx))
        if st != PG_OK:
            raise PgError(st, f"pg_create(device={device}) failed")
        self.ctx = ctx

    def close(self) -> None:
        if self.ctx:
            self.lib.pg_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        return self.lib.pg_last_error(self.ctx).decode()

    def _check(self, st: int) -> None:
        if st != PG_OK:
            raise PgError(st, self.last_error())

    def mul_limbs(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        out = np.zeros(max(len(a) + len(b), 1), dtype=np.uint64)
        n = ctypes.c_size_t(0)
        self._check(self.lib.pg_mul(self.ctx, _ptr(a), len(a), _ptr(b), len(b), _ptr(out), len(out),
                                    ctypes.byref(n)))
        return out[: n.value]

    def sqr_limbs(self, a: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.uint64)
        out = np.zeros(max(2 * len(a), 1), dtype=np.uint64)
        n = ctypes.c_size_t(0)
        self._check(self.lib.pg_sqr(self.ctx, _ptr(a), len(a), _ptr(out), len(out), ctypes.byref(n)))
        return out[: n.value]

    def mul(self, a: int, b: int) -> int:
        """Signed product like GmpMultiplier::multiply: sign handled here, magnitudes on the GPU."""
        sign = (-1 if a < 0 else 1) * (-1 if b < 0 else 1)
        r = limbs_to_int(self.mul_limbs(int_to_limbs(a), int_to_limbs(b)))
        return -r if sign < 0 else r

    def sqr(self, a: int) -> int:
        return limbs_to_int(self.sqr_limbs(int_to_limbs(a)))

    # -------------------------------------------------- device-resident finish
    def recip_floor(self, r: int) -> int:
        """floor(2^(2k) / r), k = r.bit_length() (pg_recip_floor)."""
        a = int_to_limbs(r)
        out = np.zeros(len(a) + 2, dtype=np.uint64)
        n = ctypes.c_size_t(0)
        self._check(self.lib.pg_recip_floor(self.ctx, _ptr(a), len(a), _ptr(out), len(out), ctypes.byref(n)))
        return limbs_to_int(out[: n.value])

    def mul_wrap(self, a: int, b: int, logl: int) -> int:
        """a * b mod (2^(32 * 2^logl) - 1) for a, b >= 0 of at most 2^(logl - 1) limbs (pg_mul_wrap)."""
        aa, bb = int_to_limbs(a), int_to_limbs(b)
        cap = (1 << (logl - 1)) + 2
        out = np.zeros(cap, dtype=np.uint64)
        n = ctypes.c_size_t()
        self._check(self.lib.pg_mul_wrap(self.ctx, _ptr(aa), len(aa), _ptr(bb), len(bb), logl, _ptr(out), cap,
                                         ctypes.byref(n)))
        return limbs_to_int(out[: n.value])

    def sqrt_scaled(self, a: int, s: int) -> int:
        """floor(sqrt(a) * 2^s) (pg_sqrt_scaled)."""
        out = np.zeros(s // 64 + 4, dtype=np.uint64)
        n = ctypes.c_size_t(0)
        self._check(self.lib.pg_sqrt_scaled(self.ctx, a, s, _ptr(out), len(out), ctypes.byref(n)))
        return limbs_to_int(out[: n.value])

    def to_decimal(self, x: int, ndigits: int) -> str:
        """The ndigits decimal digits of x (leading zeros kept) (pg_to_decimal)."""
        a = int_to_limbs(x)
        buf = ctypes.create_string_buffer(max(ndigits, 1))
        self._check(self.lib.pg_to_decimal(self.ctx, _ptr(a), len(a), ndigits, buf))
        return buf.raw[:ndigits].decode()

    def pi_finish(self, q: int, r: int, digits: int) -> str:
        """"3." + digits of pi from the series root Q, R (pg_pi_finish)."""
        qa, ra = int_to_limbs(q), int_to_limbs(r)
        buf = ctypes.create_string_buffer(digits + 2)
        self._check(self.lib.pg_pi_finish(self.ctx, _ptr(qa), len(qa), _ptr(ra), len(ra), digits, buf))
        return buf.raw[: digits + 2].decode()

    def pi(self, digits: int, seconds: Optional[list] = None) -> bytes:
        """"3." + digits of pi computed entirely on the device (pg_pi)."""
        buf = ctypes.create_string_buffer(digits + 2)
        t = (ctypes.c_double * 4)()
        self._check(self.lib.pg_pi(self.ctx, digits, buf, t))
        if seconds is not None:
            seconds[:] = list(t)
        return buf.raw[: digits + 2]

    def bs(self, a: int, b: int) -> tuple:
        """(P, Q, R) of the term range [a, b) by the device splitting (pg_bs), as signed ints."""
        cap = 64 + 8 * (b - a)
        bufs = [np.zeros(cap, dtype=np.uint64) for _ in range(3)]
        n = (ctypes.c_size_t * 3)()
        sg = (ctypes.c_int * 3)()
        self._check(self.lib.pg_bs(self.ctx, a, b, bufs[0].ctypes.data, _ptr(bufs[1]), _ptr(bufs[2]), cap, n, sg))
        return tuple(sg[k] * limbs_to_int(bufs[k][: n[k]]) for k in range(3))

    # -------------------------------------------------- checkpoints
    def bs_checkpointed(self, a: int, b: int, directory: str) -> tuple:
        """((P, Q, R), report) for the term range [a, b) resumed from and saved to `directory`
        (pg_bs_checkpointed), the values as signed ints."""
        cap = 64 + 8 * (b - a)
        bufs = [np.zeros(cap, dtype=np.uint64) for _ in range(3)]
        n = (ctypes.c_size_t * 3)()
        sg = (ctypes.c_int * 3)()
        rep = PgCkptReport()
        self._check(self.lib.pg_bs_checkpointed(self.ctx, a, b, directory.encode(), bufs[0].ctypes.data,
                                                _ptr(bufs[1]), _ptr(bufs[2]), cap, n, sg, ctypes.byref(rep)))
        vals = tuple(sg[k] * limbs_to_int(bufs[k][: n[k]]) for k in range(3))
        return vals, rep.as_dict()

    def pi_checkpointed(self, digits: int, directory: str, seconds: Optional[list] = None) -> tuple:
        """("3." + digits of pi, report) with the reference's --checkpoint behaviour
        (pg_pi_checkpointed)."""
        buf = ctypes.create_string_buffer(digits + 2)
        t = (ctypes.c_double * 4)()
        rep = PgCkptReport()
        self._check(self.lib.pg_pi_checkpointed(self.ctx, digits, directory.encode(), buf, t, ctypes.byref(rep)))
        if seconds is not None:
            seconds[:] = list(t)
        return buf.raw[: digits + 2], rep.as_dict()

    # -------------------------------------------------- autotuner
    def tune(self, lo: int, hi: int) -> list:
        """Run pg_tune over transform lengths 2^lo .. 2^hi; returns the winning times (us)."""
        out = (ctypes.c_double * (hi - lo + 1))()
        self._check(self.lib.pg_tune(self.ctx, lo, hi, out))
        return list(out)

    def tune_save(self, path: str) -> None:
        self._check(self.lib.pg_tune_save(self.ctx, path.encode()))

    def tune_load(self, path: str) -> None:
        self._check(self.lib.pg_tune_load(self.ctx, path.encode()))

    # -------------------------------------------------- device buffers and batches
    def buffer(self, limbs) -> "DeviceBuffer":
        """A pg_buf holding `limbs` (numpy uint64 array or int), capacity at least 1 limb."""
        a = limbs if isinstance(limbs, np.ndarray) else int_to_limbs(limbs)
        a = np.ascontiguousarray(a, dtype=np.uint64)
        return DeviceBuffer(self, max(len(a), 1), a)

    def mul_batch(self, jobs: list) -> list:
        """Products of a list of jobs through pg_mul_batch. Each job is (a, b) for a*b, (a, None)
        for a*a, or (a, b, c, d, acc) for a*b + acc*c*d (d may be None for c*c); operands are ints
        (magnitudes) or limb arrays. Returns the results as Python ints."""
        keep, cj, outs = [], [], []
        for j in jobs:
            a, b = j[0], j[1]
            c, d, acc = (j[2], j[3], j[4]) if len(j) > 2 else (None, None, 0)
            ba = self.buffer(a)
            bb = self.buffer(b) if b is not None else None
            bc = self.buffer(c) if acc else None
            bd = self.buffer(d) if acc and d is not None else None
            na, nb = ba.len, (bb.len if bb else ba.len)
            nc = bc.len if bc else 0
            nd = (bd.len if bd else nc) if acc else 0
            top = max(na + nb, nc + nd) + (1 if acc > 0 else 0)
            bo = DeviceBuffer(self, max(top, 1), None)
            keep += [x for x in (ba, bb, bc, bd, bo) if x is not None]
            pj = PgJob(ba.ptr, na, bb.ptr if bb else None, nb, bc.ptr if bc else None, nc,
                       bd.ptr if bd else None, nd if bd else 0, acc, bo.ptr, bo.cap)
            if acc and bd is None:
                pj.nd = 0
            cj.append(pj)
            outs.append((bo, top))
        arr = (PgJob * len(cj))(*cj)
        self._check(self.lib.pg_mul_batch(self.ctx, arr, len(cj)))
        res = []
        for bo, top in outs:
            bo.set_len(top)
            res.append(limbs_to_int(bo.download()))
        for x in keep:
            x.free()
        return res


# ------------------------------------------------------------------ checkpoint files (no device)
def _ckpt_check(st: int, what: str) -> None:
    if st != PG_OK:
        raise PgError(st, what)


def ckpt_write_bs(path: str, P: int, Q: int, R: int) -> None:
    """Write bs_<a>_<b>.ckpt content for signed P, Q, R (pg_ckpt_write_bs)."""
    lib = load_library()
    arrs = [int_to_limbs(abs(v)) for v in (P, Q, R)]
    ptrs = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in arrs])
    n = (ctypes.c_size_t * 3)(*[len(a) if v else 0 for a, v in zip(arrs, (P, Q, R))])
    sg = (ctypes.c_int * 3)(*[(v > 0) - (v < 0) for v in (P, Q, R)])
    _ckpt_check(lib.pg_ckpt_write_bs(path.encode(), ptrs, n, sg), f"pg_ckpt_write_bs {path}")


def ckpt_read_bs(path: str) -> tuple:
    """Signed (P, Q, R) from a splitting checkpoint file (pg_ckpt_read_bs)."""
    lib = load_library()
    n = (ctypes.c_size_t * 3)()
    sg = (ctypes.c_int * 3)()
    _ckpt_check(lib.pg_ckpt_read_bs(path.encode(), None, 0, n, sg), f"pg_ckpt_read_bs {path}")
    cap = max(1, max(n))
    arrs = [np.zeros(cap, dtype=np.uint64) for _ in range(3)]
    ptrs = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in arrs])
    _ckpt_check(lib.pg_ckpt_read_bs(path.encode(), ptrs, cap, n, sg), f"pg_ckpt_read_bs {path}")
    return tuple(sg[k] * limbs_to_int(arrs[k][: n[k]]) for k in range(3))


def ckpt_write_pi_int(path: str, x: int) -> None:
    """Write a pi_int_<digits>.ckpt file for x >= 0 (pg_ckpt_write_pi_int)."""
    a = int_to_limbs(x)
    _ckpt_check(load_library().pg_ckpt_write_pi_int(path.encode(), _ptr(a), len(a) if x else 0),
                f"pg_ckpt_write_pi_int {path}")


def ckpt_read_pi_int(path: str) -> int:
    """The integer of a pi_int checkpoint file (pg_ckpt_read_pi_int)."""
    lib = load_library()
    n = ctypes.c_size_t()
    _ckpt_check(lib.pg_ckpt_read_pi_int(path.encode(), None, 0, ctypes.byref(n)), f"pg_ckpt_read_pi_int {path}")
    a = np.zeros(max(1, n.value), dtype=np.uint64)
    _ckpt_check(lib.pg_ckpt_read_pi_int(path.encode(), a.ctypes.data, len(a), ctypes.byref(n)),
                f"pg_ckpt_read_pi_int {path}")
    return limbs_to_int(a[: n.value])


class DeviceBuffer:
    """A pg_buf: `cap` limbs of device memory owned by the library, with a length."""

    def __init__(self, eng: Engine, cap: int, data: Optional[np.ndarray]):
        self.eng, self.cap = eng, cap
        h = ctypes.c_void_p()
        eng._check(eng.lib.pg_buf_alloc(eng.ctx, cap, ctypes.byref(h)))
        self.h = h
        if data is not None and len(data):
            eng._check(eng.lib.pg_buf_upload(eng.ctx, h, _ptr(data), len(data)))

    @property
    def ptr(self) -> int:
        return self.eng.lib.pg_buf_device(self.h)

    @property
    def len(self) -> int:
        return self.eng.lib.pg_buf_len(self.h)

    def set_len(self, n: int) -> None:
        self.eng._check(self.eng.lib.pg_buf_set_len(self.h, n))

    def download(self) -> np.ndarray:
        out = np.zeros(max(self.len, 1), dtype=np.uint64)
        n = ctypes.c_size_t(0)
        self.eng._check(self.eng.lib.pg_buf_download(self.eng.ctx, self.h, _ptr(out), len(out), ctypes.byref(n)))
        return out[: n.value]

    def free(self) -> None:
        if self.h:
            self.eng.lib.pg_buf_free(self.eng.ctx, self.h)
            self.h = None
