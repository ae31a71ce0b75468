"""Test infrastructure only: ctypes bindings for the oracle libraries.

* ``Oracle`` -- the plain-C restatement ``oracle/leco_oracle.c``
  (``oracle/_build/liboracle.so``).
* ``Reference`` -- the unmodified reference codec headers compiled by
  ``oracle/Makefile`` into ``oracle/_ref/libleco_ref.so`` (present only when it
  was built where the reference sources exist; the built file travels with the
  repository snapshot).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use this
module; the product never imports it.

Codec ids follow the product's C ABI: 0 LeCo linear, 1 FOR, 2 Delta, 3 LeCo
degree-2 polynomial.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libleco_ref.so")
# The reference checkout sits beside this repository unless LECO_REFERENCE_ROOT names it.
REF_ROOT = os.environ.get("LECO_REFERENCE_ROOT", os.path.abspath(os.path.join(HERE, "..", "..", "reference")))

LECO, FOR, DELTA, POLY2 = 0, 1, 2, 3
_P = ctypes.c_void_p
_SZ = ctypes.c_size_t


def build(force: bool = False) -> None:
    """Compiles the oracle libraries with oracle/Makefile (gcc only)."""
    if force or not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-s", "-C", HERE, "_build/liboracle.so"])
    if os.path.isdir(os.path.join(REF_ROOT, "headers")):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"LECO_REFERENCE_ROOT={REF_ROOT}"])


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _dtype(s: int):
    return np.uint64 if s == 8 else np.uint32


def worst_case_bytes(n: int, s: int, bs: int) -> int:
    nb = (n + bs - 1) // bs
    return n * s + nb * 64 + 64


class Oracle:
    """The plain-C restatement of the reference algorithm."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        self.L = L
        for name in ("oracle_leco_encode", "oracle_for_encode", "oracle_delta_encode", "oracle_poly2_encode"):
            getattr(L, name).restype = _SZ
            getattr(L, name).argtypes = [_P, ctypes.c_int, _SZ, _P]
        for name in ("oracle_leco_decode", "oracle_for_decode", "oracle_delta_decode", "oracle_poly2_decode"):
            getattr(L, name).restype = _SZ
            getattr(L, name).argtypes = [_P, ctypes.c_int, _SZ, _P, ctypes.c_int]
        for name in ("oracle_leco_random", "oracle_for_random", "oracle_delta_random", "oracle_poly2_random"):
            getattr(L, name).restype = ctypes.c_uint64
            getattr(L, name).argtypes = [_P, ctypes.c_int, ctypes.c_int]
        L.oracle_column_encode.restype = _SZ
        L.oracle_column_encode.argtypes = [ctypes.c_int, _P, ctypes.c_int, _SZ, ctypes.c_uint32, _P, _P]
        L.oracle_column_decode.restype = None
        L.oracle_column_decode.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int, _SZ, ctypes.c_uint32, _P]
        L.oracle_column_random.restype = None
        L.oracle_column_random.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_uint32, _P, _SZ, _P]
        L.oracle_column_sum.restype = ctypes.c_uint64
        L.oracle_column_sum.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int, _SZ, ctypes.c_uint32, _P]
        L.oracle_varseg_encode.restype = _SZ
        L.oracle_varseg_encode.argtypes = [_P, ctypes.c_uint32, ctypes.c_uint32, _P]
        L.oracle_varseg_decode.restype = _SZ
        L.oracle_varseg_decode.argtypes = [_P, _SZ, _P]
        L.oracle_varseg_random.restype = ctypes.c_uint64
        L.oracle_varseg_random.argtypes = [_P, ctypes.c_uint64]
        L.oracle_lr_fit.restype = None
        L.oracle_lr_fit.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P, _P]
        L.oracle_poly2_fit.restype = None
        L.oracle_poly2_fit.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P]
        L.oracle_leco_filter.restype = _SZ
        L.oracle_leco_filter.argtypes = [_P, ctypes.c_int, _SZ, ctypes.c_uint64, ctypes.c_uint32, _P]
        L.oracle_for_filter.restype = _SZ
        L.oracle_for_filter.argtypes = [_P, ctypes.c_int, _SZ, ctypes.c_uint64, ctypes.c_uint32, _P]
        L.oracle_leco_filter_close.restype = _SZ
        L.oracle_leco_filter_close.argtypes = [_P, ctypes.c_int, _SZ, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32,
                                               ctypes.c_uint32, _P, ctypes.c_int, ctypes.c_uint64]
        L.oracle_for_filter_close.restype = _SZ
        L.oracle_for_filter_close.argtypes = [_P, ctypes.c_int, _SZ, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32,
                                              ctypes.c_uint32, _P]
        L.oracle_close_window_start.restype = None
        L.oracle_close_window_start.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                                ctypes.c_int, _P, _P]
        L.oracle_legacy_encode.restype = _SZ
        L.oracle_legacy_encode.argtypes = [_P, _SZ, _P, _P, _P]
        L.oracle_legacy_decode.restype = None
        L.oracle_legacy_decode.argtypes = [_P, _SZ, _P, ctypes.c_int]
        L.oracle_legacy_random.restype = ctypes.c_uint32
        L.oracle_legacy_random.argtypes = [_P, ctypes.c_int]
        L.oracle_column_zonemap.restype = None
        L.oracle_column_zonemap.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int, _SZ, ctypes.c_uint32, _P, _P, _P]
        L.oracle_column_filter.restype = _SZ
        L.oracle_column_filter.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int, _SZ, ctypes.c_uint32, ctypes.c_uint64, _P, _P]
        L.oracle_column_filter_close.restype = _SZ
        L.oracle_column_filter_close.argtypes = [ctypes.c_int, _P, _P, ctypes.c_int, _SZ, ctypes.c_uint32, ctypes.c_uint64,
                                                 ctypes.c_uint64, ctypes.c_uint64, _P, _P, ctypes.c_int, ctypes.c_uint64]

    _ENC = ("oracle_leco_encode", "oracle_for_encode", "oracle_delta_encode", "oracle_poly2_encode")
    _DEC = ("oracle_leco_decode", "oracle_for_decode", "oracle_delta_decode", "oracle_poly2_decode")
    _RA = ("oracle_leco_random", "oracle_for_random", "oracle_delta_random", "oracle_poly2_random")

    # -- one block --------------------------------------------------------
    def encode_block(self, codec: int, data: np.ndarray) -> bytes:
        data = np.ascontiguousarray(data)
        s = data.dtype.itemsize
        out = np.zeros(len(data) * s + 128, np.uint8)
        nbytes = getattr(self.L, self._ENC[codec])(_ptr(data), s, len(data), _ptr(out))
        return out[:nbytes].tobytes()

    def decode_block(self, codec: int, block: bytes, n: int, s: int, strict_raw: int = 1) -> np.ndarray:
        buf = np.frombuffer(block + b"\0" * 32, np.uint8).copy()
        out = np.zeros(max(n, 2), _dtype(s))
        getattr(self.L, self._DEC[codec])(_ptr(buf), s, n, _ptr(out), strict_raw)
        return out[:n]

    def random_block(self, codec: int, block: bytes, k: int, s: int) -> int:
        buf = np.frombuffer(block + b"\0" * 32, np.uint8).copy()
        return int(getattr(self.L, self._RA[codec])(_ptr(buf), s, k))

    def lr_fit(self, data: np.ndarray):
        t = np.zeros(2, np.float64)
        self.L.oracle_lr_fit(_ptr(data), data.dtype.itemsize, len(data), _ptr(t[:1]), _P(t.ctypes.data + 8))
        return float(t[0]), float(t[1])

    def poly2_fit(self, data: np.ndarray):
        a = np.zeros(3, np.float64)
        self.L.oracle_poly2_fit(_ptr(data), data.dtype.itemsize, len(data), _ptr(a))
        return a

    # -- whole column -----------------------------------------------------
    def encode_column(self, codec: int, data: np.ndarray, bs: int):
        data = np.ascontiguousarray(data)
        s, n = data.dtype.itemsize, len(data)
        nb = (n + bs - 1) // bs
        out = np.zeros(worst_case_bytes(n, s, bs), np.uint8)
        off = np.zeros(nb + 1, np.uint64)
        total = self.L.oracle_column_encode(codec, _ptr(data), s, n, bs, _ptr(out), _ptr(off))
        return out[:total].copy(), off

    def decode_column(self, codec: int, payload: np.ndarray, offsets: np.ndarray, n: int, s: int, bs: int):
        pay = np.concatenate([payload, np.zeros(64, np.uint8)])
        out = np.zeros(n, _dtype(s))
        self.L.oracle_column_decode(codec, _ptr(pay), _ptr(offsets), s, n, bs, _ptr(out))
        return out

    def random_column(self, codec: int, payload: np.ndarray, offsets: np.ndarray, s: int, bs: int, idx: np.ndarray):
        pay = np.concatenate([payload, np.zeros(64, np.uint8)])
        idx = np.ascontiguousarray(idx, np.uint64)
        out = np.zeros(len(idx), _dtype(s))
        self.L.oracle_column_random(codec, _ptr(pay), _ptr(offsets), s, bs, _ptr(idx), len(idx), _ptr(out))
        return out

    # -- legacy u32 format (piecewise_fix_op_max) ---------------------------
    def legacy_encode_block(self, data: np.ndarray):
        """(image bytes, diff_plus bool[n], diff_minus bool[n])."""
        data = np.ascontiguousarray(data, np.uint32)
        out = np.zeros(len(data) * 4 + 64, np.uint8)
        dp, dm = np.zeros(len(data), np.uint8), np.zeros(len(data), np.uint8)
        nb = self.L.oracle_legacy_encode(_ptr(data), len(data), _ptr(out), _ptr(dp), _ptr(dm))
        return out[:nb].tobytes(), dp.astype(bool), dm.astype(bool)

    def legacy_decode_block(self, block: bytes, n: int, add_pred: bool = False) -> np.ndarray:
        buf = np.frombuffer(block + b"\0" * 32, np.uint8).copy()
        out = np.zeros(max(n, 1), np.uint32)
        self.L.oracle_legacy_decode(_ptr(buf), n, _ptr(out), int(add_pred))
        return out[:n]

    def legacy_random(self, block: bytes, k: int) -> int:
        buf = np.frombuffer(block + b"\0" * 32, np.uint8).copy()
        return int(self.L.oracle_legacy_random(_ptr(buf), k))

    # -- predicate pushdown ------------------------------------------------
    def zonemap(self, codec: int, payload: np.ndarray, offsets: np.ndarray, n: int, s: int, bs: int):
        """Per-block (min, max) of the decoded values, as uint64 arrays."""
        pay = np.concatenate([payload, np.zeros(64, np.uint8)])
        nb = (n + bs - 1) // bs
        scratch = np.zeros(max(n, 1), _dtype(s))
        zmin, zmax = np.zeros(nb, np.uint64), np.zeros(nb, np.uint64)
        self.L.oracle_column_zonemap(codec, _ptr(pay), _ptr(offsets), s, n, bs, _ptr(scratch), _ptr(zmin), _ptr(zmax))
        return zmin, zmax

    def block_filter(self, codec: int, block: bytes, n: int, s: int, filt: int, block_start: int = 0) -> np.ndarray:
        buf = np.frombuffer(block + b"\0" * 32, np.uint8).copy()
        out = np.zeros(n + 1, np.uint32)
        fn = self.L.oracle_leco_filter if codec == LECO else self.L.oracle_for_filter
        c = fn(_ptr(buf), s, n, filt, block_start, _ptr(out))
        return out[:c].copy()

    def block_filter_close(self, codec: int, block: bytes, n: int, s: int, f1: int, f2: int, base: int,
                           block_start: int = 0, overwrite: bool = False, max_periods: int = 0, out_len: int | None = None):
        """(count, out buffer); count -1 when max_periods windows were reached."""
        buf = np.frombuffer(block + b"\0" * 32, np.uint8).copy()
        out = np.zeros(out_len if out_len is not None else 4 * n + 2, np.uint32)
        if codec == LECO:
            c = self.L.oracle_leco_filter_close(_ptr(buf), s, n, f1, f2, base, block_start, _ptr(out), int(overwrite), max_periods)
        else:
            c = self.L.oracle_for_filter_close(_ptr(buf), s, n, f1, f2, base, block_start, _ptr(out))
        return (-1 if c == 2**64 - 1 else c), out

    def close_window_start(self, zmin: int, f1: int, f2: int, base: int, s: int):
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        self.L.oracle_close_window_start(zmin, f1, f2, base, s, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def filter_column(self, codec: int, payload: np.ndarray, offsets: np.ndarray, n: int, s: int, bs: int,
                      filt: int, zmax: np.ndarray | None = None) -> np.ndarray:
        """Indices (uint32) of the values above `filt`, blocks in order."""
        pay = np.concatenate([payload, np.zeros(64, np.uint8)])
        out = np.zeros(n + 1, np.uint32)
        zp = _ptr(np.ascontiguousarray(zmax, np.uint64)) if zmax is not None else None
        c = self.L.oracle_column_filter(codec, _ptr(pay), _ptr(offsets), s, n, bs, filt, zp, _ptr(out))
        return out[:c].copy()

    def filter_close_column(self, codec: int, payload: np.ndarray, offsets: np.ndarray, n: int, s: int, bs: int,
                            f1: int, f2: int, base: int, zmin: np.ndarray | None = None, overwrite: bool = False,
                            max_periods: int = 0, out_len: int | None = None):
        """(count, out buffer) of the close-range filter; out_len sizes the
        buffer (default 4n + nblocks + 1).  count is -1 when a block reached
        max_periods windows."""
        pay = np.concatenate([payload, np.zeros(64, np.uint8)])
        nb = (n + bs - 1) // bs
        out = np.zeros(out_len if out_len is not None else 4 * n + nb + 1, np.uint32)
        zm = np.ascontiguousarray(zmin, np.uint64) if zmin is not None else None
        c = self.L.oracle_column_filter_close(codec, _ptr(pay), _ptr(offsets), s, n, bs, f1, f2, base,
                                              _ptr(zm) if zm is not None else None, _ptr(out), int(overwrite), max_periods)
        return (-1 if c == 2**64 - 1 else c), out

    # -- variable-length segments ----------------------------------------
    def varseg_encode(self, array: np.ndarray, start: int, end: int) -> bytes:
        out = np.zeros((end - start + 1) * 8 + 64, np.uint8)
        nbytes = self.L.oracle_varseg_encode(_ptr(array), start, end, _ptr(out))
        return out[:nbytes].tobytes()

    def varseg_decode(self, seg: bytes, length: int) -> np.ndarray:
        buf = np.frombuffer(seg + b"\0" * 32, np.uint8).copy()
        out = np.zeros(max(length, 2), np.uint64)
        self.L.oracle_varseg_decode(_ptr(buf), length, _ptr(out))
        return out[:length]

    def varseg_random(self, seg: bytes, g: int) -> int:
        buf = np.frombuffer(seg + b"\0" * 32, np.uint8).copy()
        return int(self.L.oracle_varseg_random(_ptr(buf), g))


class Reference:
    """The reference's own codec classes (compiled headers), via ref_wrap.cpp."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        self.L = L
        for t, ct in (("u32", ctypes.c_uint32), ("u64", ctypes.c_uint64)):
            f = getattr(L, f"ref_encode_block_{t}"); f.restype = _SZ; f.argtypes = [ctypes.c_int, _P, _SZ, _P]
            f = getattr(L, f"ref_decode_block_{t}"); f.restype = None; f.argtypes = [ctypes.c_int, _P, _SZ, _P]
            f = getattr(L, f"ref_random_{t}"); f.restype = ct; f.argtypes = [ctypes.c_int, _P, ctypes.c_int]
            f = getattr(L, f"ref_column_encode_{t}"); f.restype = _SZ; f.argtypes = [ctypes.c_int, _P, _SZ, ctypes.c_uint32, _P, _P]
            f = getattr(L, f"ref_column_encode_mt_{t}"); f.restype = _SZ; f.argtypes = [ctypes.c_int, _P, _SZ, ctypes.c_uint32, _P, _P, ctypes.c_int]
            f = getattr(L, f"ref_column_decode_{t}"); f.restype = None; f.argtypes = [ctypes.c_int, _P, _P, _SZ, ctypes.c_uint32, _P, ctypes.c_int]
            f = getattr(L, f"ref_column_random_{t}"); f.restype = None; f.argtypes = [ctypes.c_int, _P, _P, ctypes.c_uint32, _P, _SZ, _P, ctypes.c_int]
        L.ref_varlen_encode_u64.restype = _P
        L.ref_varlen_encode_u64.argtypes = [_P, _SZ, ctypes.c_int, ctypes.c_int64]
        L.ref_varlen_segments.restype = _SZ
        L.ref_varlen_segments.argtypes = [_P]
        L.ref_varlen_export.restype = _SZ
        L.ref_varlen_export.argtypes = [_P, _P, _P, _P]
        L.ref_varlen_decode.restype = None
        L.ref_varlen_decode.argtypes = [_P, _SZ, _P]
        L.ref_varlen_random.restype = None
        L.ref_varlen_random.argtypes = [_P, _P, _SZ, _P]
        L.ref_varlen_free.restype = None
        L.ref_varlen_free.argtypes = [_P]
        L.ref_legacy_encode_block.restype = _SZ
        L.ref_legacy_encode_block.argtypes = [_P, _SZ, _P, _P, _P]
        L.ref_legacy_decode_block.restype = None
        L.ref_legacy_decode_block.argtypes = [_P, _SZ, _P]
        L.ref_legacy_random.restype = ctypes.c_uint32
        L.ref_legacy_random.argtypes = [_P, ctypes.c_int]
        for t, ct in (("u32", ctypes.c_uint32), ("u64", ctypes.c_uint64)):
            f = getattr(L, f"ref_column_filter_{t}"); f.restype = _SZ
            f.argtypes = [ctypes.c_int, _P, _P, _SZ, ctypes.c_uint32, ct, _P, _P]
            f = getattr(L, f"ref_column_filter_close_{t}"); f.restype = _SZ
            f.argtypes = [ctypes.c_int, _P, _P, _SZ, ctypes.c_uint32, ct, ct, ct, _P, _P]
            f = getattr(L, f"ref_block_filter_{t}"); f.restype = _SZ
            f.argtypes = [ctypes.c_int, _P, _SZ, ctypes.c_uint32, ctypes.c_int, ct, _P]
            f = getattr(L, f"ref_block_filter_close_{t}"); f.restype = _SZ
            f.argtypes = [ctypes.c_int, _P, _SZ, ctypes.c_uint32, ctypes.c_int, ct, ct, ctypes.c_int, _P]
            f = getattr(L, f"ref_close_window_start_{t}"); f.restype = None
            f.argtypes = [ct, ct, ct, ct, _P, _P]

    @staticmethod
    def _t(s):
        return "u64" if s == 8 else "u32"

    def encode_block(self, codec: int, data: np.ndarray) -> bytes:
        data = np.ascontiguousarray(data)
        s = data.dtype.itemsize
        out = np.zeros(len(data) * s * 4 + 128, np.uint8)
        nbytes = getattr(self.L, f"ref_encode_block_{self._t(s)}")(codec, _ptr(data), len(data), _ptr(out))
        return out[:nbytes].tobytes()

    def decode_block(self, codec: int, block: bytes, n: int, s: int) -> np.ndarray:
        buf = np.frombuffer(block + b"\0" * 32, np.uint8).copy()
        out = np.zeros(max(n, 2) + 64, _dtype(s))
        getattr(self.L, f"ref_decode_block_{self._t(s)}")(codec, _ptr(buf), n, _ptr(out))
        return out[:n]

    def random_block(self, codec: int, block: bytes, k: int, s: int) -> int:
        buf = np.frombuffer(block + b"\0" * 32, np.uint8).copy()
        return int(getattr(self.L, f"ref_random_{self._t(s)}")(codec, _ptr(buf), k))

    def encode_column(self, codec: int, data: np.ndarray, bs: int, threads: int = 1):
        data = np.ascontiguousarray(data)
        s, n = data.dtype.itemsize, len(data)
        nb = (n + bs - 1) // bs
        out = np.empty(worst_case_bytes(n, s, bs) + n * s, np.uint8)
        off = np.zeros(nb + 1, np.uint64)
        if threads > 1:
            total = getattr(self.L, f"ref_column_encode_mt_{self._t(s)}")(codec, _ptr(data), n, bs, _ptr(out), _ptr(off),
                                                                          threads)
        else:
            total = getattr(self.L, f"ref_column_encode_{self._t(s)}")(codec, _ptr(data), n, bs, _ptr(out), _ptr(off))
        return out[:total].copy(), off

    @staticmethod
    def pad(payload: np.ndarray) -> np.ndarray:
        """The payload followed by the 64 zero bytes the block readers may touch."""
        return np.concatenate([payload, np.zeros(64, np.uint8)])

    def decode_column(self, codec: int, payload: np.ndarray, offsets: np.ndarray, n: int, s: int, bs: int, threads: int = 1,
                      out: np.ndarray | None = None, padded: bool = False):
        """Bulk decode of a column (per block decodeArray8).  `padded`: the payload
        already carries pad()'s 64 bytes; `out` (>= n + 64 values) is reused."""
        pay = payload if padded else self.pad(payload)
        if out is None:
            out = np.zeros(n + 64, _dtype(s))
        getattr(self.L, f"ref_column_decode_{self._t(s)}")(codec, _ptr(pay), _ptr(offsets), n, bs, _ptr(out), threads)
        return out[:n]

    def random_column(self, codec: int, payload: np.ndarray, offsets: np.ndarray, s: int, bs: int, idx: np.ndarray, threads: int = 1,
                      out: np.ndarray | None = None, padded: bool = False):
        """randomdecodeArray8 per index (global indices)."""
        pay = payload if padded else self.pad(payload)
        idx = np.ascontiguousarray(idx, np.uint64)
        if out is None:
            out = np.zeros(len(idx), _dtype(s))
        getattr(self.L, f"ref_column_random_{self._t(s)}")(codec, _ptr(pay), _ptr(offsets), bs, _ptr(idx), len(idx), _ptr(out), threads)
        return out[:len(idx)]

    # -- legacy u32 format (piecewise_fix_op_max) ---------------------------
    def legacy_encode_block(self, data: np.ndarray):
        data = np.ascontiguousarray(data, np.uint32)
        out = np.zeros(len(data) * 4 + 1000, np.uint8)
        dp, dm = np.zeros(len(data), np.uint8), np.zeros(len(data), np.uint8)
        nb = self.L.ref_legacy_encode_block(_ptr(data), len(data), _ptr(out), _ptr(dp), _ptr(dm))
        return out[:nb].tobytes(), dp.astype(bool), dm.astype(bool)

    def legacy_decode_block(self, block: bytes, n: int) -> np.ndarray:
        buf = np.frombuffer(block + b"\0" * 64, np.uint8).copy()
        out = np.zeros(n + 64, np.uint32)
        self.L.ref_legacy_decode_block(_ptr(buf), n, _ptr(out))
        return out[:n]

    def legacy_random(self, block: bytes, k: int) -> int:
        buf = np.frombuffer(block + b"\0" * 64, np.uint8).copy()
        return int(self.L.ref_legacy_random(_ptr(buf), k))

    # -- predicate pushdown (the filter experiments' loops) -----------------
    def filter_column(self, codec: int, payload: np.ndarray, offsets: np.ndarray, n: int, s: int, bs: int,
                      filt: int, zmax: np.ndarray | None = None) -> np.ndarray:
        pay = np.concatenate([payload, np.zeros(64, np.uint8)])
        out = np.zeros(n + 64, np.uint32)
        zp = _ptr(np.ascontiguousarray(zmax, np.uint64)) if zmax is not None else None
        c = getattr(self.L, f"ref_column_filter_{self._t(s)}")(codec, _ptr(pay), _ptr(offsets), n, bs, filt, zp, _ptr(out))
        return out[:c].copy()

    def block_filter(self, codec: int, block: bytes, n: int, s: int, filt: int, bs: int, block_id: int):
        """(count, out buffer) of one block's filter_range."""
        buf = np.frombuffer(block + b"\0" * 64, np.uint8).copy()
        out = np.zeros(n + 64, np.uint32)
        c = getattr(self.L, f"ref_block_filter_{self._t(s)}")(codec, _ptr(buf), n, bs, block_id, filt, _ptr(out))
        return c, out

    def block_filter_close(self, codec: int, block: bytes, n: int, s: int, f1: int, f2: int, base: int, bs: int,
                           block_id: int):
        """(count, out buffer) of one block's filter_range_close."""
        buf = np.frombuffer(block + b"\0" * 64, np.uint8).copy()
        out = np.zeros(4 * n + 64, np.uint32)
        c = getattr(self.L, f"ref_block_filter_close_{self._t(s)}")(codec, _ptr(buf), n, bs, block_id, f1, f2, base, _ptr(out))
        return c, out

    def close_window_start(self, zmin: int, f1: int, f2: int, base: int, s: int):
        ct = ctypes.c_uint64 if s == 8 else ctypes.c_uint32
        a, b = ct(), ct()
        getattr(self.L, f"ref_close_window_start_{self._t(s)}")(zmin, f1, f2, base, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def filter_close_column(self, codec: int, payload: np.ndarray, offsets: np.ndarray, n: int, s: int, bs: int,
                            f1: int, f2: int, base: int, zmin: np.ndarray | None = None, out_len: int | None = None):
        """(count, out buffer) exactly as the reference leaves them."""
        pay = np.concatenate([payload, np.zeros(64, np.uint8)])
        nb = (n + bs - 1) // bs
        out = np.zeros(out_len if out_len is not None else 4 * n + nb + 1, np.uint32)
        zm = np.ascontiguousarray(zmin, np.uint64) if zmin is not None else None
        c = getattr(self.L, f"ref_column_filter_close_{self._t(s)}")(codec, _ptr(pay), _ptr(offsets), n, bs, f1, f2, base,
                                                                      _ptr(zm) if zm is not None else None, _ptr(out))
        return c, out

    # -- variable-length (u64) ---------------------------------------------
    def varlen_encode(self, data: np.ndarray, blocks: int, delta: int):
        """Runs the reference partitioner + segment writer; returns
        (starts[u32], byte_offsets[u64, ns+1], payload[u8])."""
        data = np.ascontiguousarray(data, np.uint64)
        h = self.L.ref_varlen_encode_u64(_ptr(data), len(data), blocks, delta)
        try:
            ns = self.L.ref_varlen_segments(h)
            starts = np.zeros(ns, np.uint32)
            off = np.zeros(ns + 1, np.uint64)
            total = self.L.ref_varlen_export(h, None, None, None)
            pay = np.zeros(total + 64, np.uint8)
            self.L.ref_varlen_export(h, _ptr(starts), _ptr(off), _ptr(pay))
            dec = np.zeros(len(data) + 64, np.uint64)
            self.L.ref_varlen_decode(h, len(data), _ptr(dec))
        finally:
            self.L.ref_varlen_free(h)
        return starts, off, pay[:total].copy(), dec[: len(data)]
