"""LeCo integer codec on B200 (sm_100a): Python host API over the C ABI.

The product is the CUDA library ``lib/libleco_b200.so`` (sources in ``csrc/``,
ABI in ``include/leco.h``).  This module binds it with ctypes and offers:

* ``Leco_int``, ``FOR_int``, ``Delta_int``, ``Leco_int_poly`` -- per-block
  mirrors of the reference classes (yhliu918/Learn-to-Compress
  headers/piecewise_fix_integer_template.h:14-338, FOR_integer_template.h:14-249,
  delta_integer_template.h:14-158, poly_fix_integer_template.h:15-292) with the
  same ``init / encodeArray8_int / decodeArray8 / randomdecodeArray8`` methods on
  host numpy buffers;
* ``encode`` / ``Column`` -- whole columns resident in device memory (torch
  tensors are used only as device allocations and for the stream handle):
  decode, range decode, random access, compressed-domain sum.

There is no CPU fallback: every call goes to the CUDA library, and importing
the library fails loudly if it was not built.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import build as _build

LINEAR, FOR, DELTA, POLY2, VARLEN, LINEAR_F32 = 0, 1, 2, 3, 4, 5
U32, U64 = 4, 8
FIT_REFERENCE, FIT_EXACT = 0, 1
PAYLOAD_SLACK = 64
MAX_BLOCK = 16384
CODEC_NAMES = {LINEAR: "leco_fix", FOR: "for_fix", DELTA: "delta_fix", POLY2: "leco_poly2", VARLEN: "leco_varlen"}

_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32
_I = ctypes.c_int

ERRORS = {
    -1: "LECO_ERR_ARG", -2: "LECO_ERR_CUDA", -3: "LECO_ERR_CORRUPT", -4: "LECO_ERR_NOMEM",
    -5: "LECO_ERR_TIMEOUT", -6: "LECO_ERR_UNSUPPORTED", -7: "LECO_ERR_CAPACITY",
}


class LecoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_LIB = None

# (name, restype, argtypes) of every entry point declared in include/leco.h
SIGNATURES = [
    ("leco_num_blocks", _U64, [_U64, _U32]),
    ("leco_max_payload_bytes", _U64, [_I, _I, _U64, _U32]),
    ("leco_encode_workspace_bytes", _U64, [_I, _I, _U64, _U32, _I]),
    ("leco_block_bytes", _U64, [_I, _I, _U32, _U32]),
    ("leco_encode", _I, [_I, _I, _P, _U64, _U32, _I, _P, _U64, _P, _P, _P, _U64, _P]),
    ("leco_encode_noalloc", _I, [_I, _I, _P, _U64, _U32, _I, _P, _U64, _P, _P, _P]),
    ("leco_encode_noalloc_max_blocks", _U64, []),
    ("leco_decode", _I, [_I, _I, _P, _P, _U64, _U32, _P, _P]),
    ("leco_decode_range", _I, [_I, _I, _P, _P, _U64, _U32, _U64, _U64, _P, _P]),
    ("leco_build_directory", _I, [_I, _I, _P, _P, _U64, _U32, _P, _P]),
    ("leco_gather", _I, [_I, _I, _P, _P, _P, _U64, _U32, _P, _U64, _P, _P]),
    ("leco_sum_workspace_bytes", _U64, [_U64, _U32]),
    ("leco_sum", _I, [_I, _I, _P, _P, _U64, _U32, _P, _P, _P]),
    ("leco_filter_workspace_bytes", _U64, [_U64, _U32]),
    ("leco_filter_range", _I, [_I, _I, _P, _P, _U64, _U32, _U64, _P, _P, _P, _U64, _P, _P, _U64, _P]),
    ("leco_filter_range_close", _I, [_I, _I, _P, _P, _U64, _U32, _U64, _U64, _U64, _P, _P, _U64, _P, _P, _U64, _P]),
    ("leco_zonemap", _I, [_I, _I, _P, _P, _U64, _U32, _P, _P, _P]),
    ("leco_block_filter", ctypes.c_int64, [_I, _I, _P, _U64, _U32, _U32, _I, _U64, _U64, _U64, _P, _U64]),
    ("leco_encode_host", _I, [_I, _I, _P, _U64, _U32, _I, _P, _U64, _P, _P]),
    ("leco_decode_host", _I, [_I, _I, _P, _P, _U64, _U32, _P]),
    ("leco_gather_host", _I, [_I, _I, _P, _P, _U64, _U32, _P, _U64, _P]),
    ("leco_block_encode", ctypes.c_int64, [_I, _I, _P, _U32, _I, _P]),
    ("leco_block_decode", _I, [_I, _I, _P, _U64, _U32, _P]),
    ("leco_block_random", _I, [_I, _I, _P, _U64, _U32, _U32, _P]),
    ("leco_thread_release", _I, []),
    ("leco_validate_host", _I, [_I, _I, _P, _U64, _P, _U64, _U32, _P]),
    ("leco_container_write", _I, [ctypes.c_char_p, _P, _P, _P, _P]),
    ("leco_container_info_read", _I, [ctypes.c_char_p, _P]),
    ("leco_container_read", _I, [ctypes.c_char_p, _P, _U64, _P, _P]),
    ("leco_container_save_device", _I, [ctypes.c_char_p, _P, _P, _P, _P, _P]),
    ("leco_container_load_device", _I, [ctypes.c_char_p, _P, _U64, _P, _P, _P]),
    ("leco_import_blocks", _I, [_P, _P, _U64, _P, _U64, _P]),
    ("leco_export_blocks", _I, [_P, _P, _U64, _P, _P]),
    ("leco_batch_create", _I, [_P, _U32, _I, _P]),
    ("leco_batch_destroy", _I, [_P]),
    ("leco_batch_total_blocks", _U64, [_P]),
    ("leco_batch_encode", _I, [_P, _P]),
    ("leco_batch_decode", _I, [_P, _P]),
    ("leco_batch_run_graph", _I, [_P, _I, _P]),
    ("leco_batch_encode_per_column", _I, [_P, _P]),
    ("leco_batch_decode_per_column", _I, [_P, _P]),
    ("leco_server_create", _I, [_P, _U32, _P, _P]),
    ("leco_server_submit", _I, [_P, _P, _P]),
    ("leco_server_wait", _I, [_P, _U64, _P]),
    ("leco_server_drain", _I, [_P]),
    ("leco_server_get_stats", _I, [_P, _P]),
    ("leco_server_reset_stats", _I, [_P]),
    ("leco_server_destroy", _I, [_P]),
    ("leco_varlen_partition", _I, [_P, _U64, _U32, ctypes.c_int64, _P, _U64, _P, _I]),
    ("leco_varlen_partition_workspace_bytes", _U64, [_U64, _U32]),
    ("leco_varlen_partition_device", _I, [_P, _U64, _U32, ctypes.c_int64, _P, _U64, _P, _P, _U64, _P]),
    ("leco_varlen_max_payload_bytes", _U64, [_U64, _U64]),
    ("leco_varlen_workspace_bytes", _U64, [_U64]),
    ("leco_varlen_max_segment", _U64, []),
    ("leco_varlen_encode", _I, [_P, _U64, _P, _U64, _U32, _I, _P, _U64, _P, _P, _U64, _P]),
    ("leco_varlen_decode", _I, [_P, _P, _P, _U64, _U64, _P, _P]),
    ("leco_varlen_gather", _I, [_P, _P, _P, _U64, _U64, _P, _U64, _P, _P]),
    ("leco_varlen_sum", _I, [_P, _P, _P, _U64, _U64, _P, _P]),
    ("leco_test_bounded_wait", _I, [_U32, _P]),
    ("leco_check", _I, [_P]),
    ("leco_last_error", ctypes.c_char_p, []),
    ("leco_version", ctypes.c_char_p, []),
]


def lib_path() -> str:
    return _build.LIB


def lib(build_if_missing: bool = True):
    """The loaded CUDA library.  Raises if it is missing and cannot be built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise FileNotFoundError(f"{path} is not built (run learn-to-compress_b200/build.py)")
        _build.build()
    L = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def _check(rc: int, what: str = "") -> int:
    if rc < 0:
        msg = lib().leco_last_error().decode()
        raise LecoError(rc, f"{what}: {msg}" if what else msg)
    return rc


def _np_ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _dtype_of(arr) -> int:
    s = arr.dtype.itemsize
    if s not in (4, 8):
        raise ValueError("values must be 32- or 64-bit unsigned integers")
    return s


def _np_dtype(s: int):
    return np.uint64 if s == 8 else np.uint32


# ---------------------------------------------------------------------------
# Per-block mirrors of the reference classes (host buffers).
# ---------------------------------------------------------------------------

class _BlockCodec:
    """Common part of the reference codec classes' per-block surface.

    ``encodeArray8_int(data, length, res, nvalue)`` writes the reference block
    image of ``data[:length]`` into the uint8 array ``res`` and returns the
    number of bytes written (the reference returns the end pointer).
    ``decodeArray8(in_, length, out, nvalue)`` decodes ``length`` values into
    ``out`` and returns it.  ``randomdecodeArray8(in_, to_find, out, nvalue)``
    returns value ``to_find`` of the block.  ``nvalue`` (the block id) and the
    unused ``out`` argument are accepted for signature parity only.
    """

    CODEC = LINEAR

    def __init__(self, dtype=np.uint64, fit_mode: int = FIT_REFERENCE):
        self.dtype = np.dtype(dtype)
        self.fit_mode = fit_mode
        self.blocks = 0
        self.block_size = 0

    def init(self, block: int, block_s: int) -> None:
        self.blocks = block
        self.block_size = block_s

    def encodeArray8_int(self, data, length: int, res: np.ndarray, nvalue: int = 0) -> int:
        data = np.ascontiguousarray(np.asarray(data, dtype=self.dtype)[:length])
        s = self.dtype.itemsize
        need = lib().leco_block_bytes(self.CODEC, s, 8 * s, length) + 64
        tmp = np.zeros(max(need, 64), np.uint8)
        nbytes = _check(lib().leco_block_encode(self.CODEC, s, _np_ptr(data), length, self.fit_mode, _np_ptr(tmp)),
                        "encodeArray8_int")
        res[:nbytes] = tmp[:nbytes]
        return nbytes

    def decodeArray8(self, in_, length: int, out: Optional[np.ndarray] = None, nvalue: int = 0) -> np.ndarray:
        buf = np.frombuffer(bytes(in_), np.uint8).copy()
        s = self.dtype.itemsize
        if out is None:
            out = np.zeros(length, self.dtype)
        o = np.zeros(length, self.dtype)
        _check(lib().leco_block_decode(self.CODEC, s, _np_ptr(buf), len(buf), length, _np_ptr(o)), "decodeArray8")
        out[:length] = o
        return out

    def randomdecodeArray8(self, in_, to_find: int, out=None, nvalue: int = 0, length: Optional[int] = None) -> int:
        buf = np.frombuffer(bytes(in_), np.uint8).copy()
        s = self.dtype.itemsize
        n = length if length is not None else (self.block_size or to_find + 1)
        v = np.zeros(1, self.dtype)
        _check(lib().leco_block_random(self.CODEC, s, _np_ptr(buf), len(buf), n, to_find, _np_ptr(v)), "randomdecodeArray8")
        return int(v[0])


class _FilterCodec(_BlockCodec):
    """The two reference classes with predicate pushdown: ``filter_range(in_,
    length, filter, out, block_id)`` and ``filter_range_close(in_, length, out,
    block_id, filter1, filter2, base)`` write indices block_id*block_size + k
    into the uint32 array ``out`` and return the count."""

    def _filter(self, in_, length, out, block_id, close, f1, f2, base):
        buf = np.frombuffer(bytes(in_), np.uint8).copy()
        s = self.dtype.itemsize
        start = block_id * self.block_size
        m = 1 << (8 * s)
        cap = length + 1
        while True:
            tmp = np.zeros(cap, np.uint32)
            c = _check(lib().leco_block_filter(self.CODEC, s, _np_ptr(buf), len(buf), length, start, close, int(f1) % m,
                                               int(f2) % m, base, _np_ptr(tmp), cap), "filter")
            if c <= cap:
                break
            cap = c
        out[:c] = tmp[:c]
        return c

    def filter_range(self, in_, length: int, filt: int, out: np.ndarray, block_id: int = 0) -> int:
        return self._filter(in_, length, out, block_id, 0, filt, 0, 0)

    def filter_range_close(self, in_, length: int, out: np.ndarray, block_id: int, filter1: int, filter2: int,
                           base: int) -> int:
        return self._filter(in_, length, out, block_id, 1, filter1, filter2, base)


class Leco_int(_FilterCodec):
    """Mirror of ``Codecset::Leco_int<T>`` (piecewise_fix_integer_template.h:14-338)."""
    CODEC = LINEAR


class FOR_int(_FilterCodec):
    """Mirror of ``Codecset::FOR_int<T>`` (FOR_integer_template.h:14-249)."""
    CODEC = FOR


class Delta_int(_BlockCodec):
    """Mirror of ``Codecset::Delta_int<T>`` (delta_integer_template.h:14-158)."""
    CODEC = DELTA


class piecewise_fix_op_max:
    """Mirror of the reference's legacy u32 codec ``Codecset::piecewise_fix_op_max``
    (piecewise_fix_op_minimize_maxerror.h:20-186).  ``encodeArray8`` writes the
    reference's block image (:45-119) and returns its byte count; the encoder's
    difference lists (mul_add_diff_set, :79-84) are not kept, because
    ``decodeArray8`` returns the stored values (the reference's own bulk decoder
    accumulates the prediction by addition and its drivers correct the difference
    with those lists afterwards, experiments/fix_int.cpp:110-117);
    ``randomdecodeArray8`` is the reference's."""

    CODEC = LINEAR_F32

    def __init__(self, fit_mode: int = FIT_REFERENCE):
        self.fit_mode = fit_mode

    def init(self, blocks: int, blocksize: int, extra: int = 0) -> None:
        self.block_num, self.block_size = blocks, blocksize

    def encodeArray8(self, in_, length: int, res: np.ndarray, nvalue: int = 0) -> int:
        data = np.ascontiguousarray(np.asarray(in_, dtype=np.uint32)[:length])
        tmp = np.zeros(int(lib().leco_block_bytes(LINEAR_F32, 4, 32, length)) + 64, np.uint8)
        nbytes = _check(lib().leco_block_encode(LINEAR_F32, 4, _np_ptr(data), length, self.fit_mode, _np_ptr(tmp)),
                        "encodeArray8")
        res[:nbytes] = tmp[:nbytes]
        return nbytes

    def decodeArray8(self, in_, length: int, out: Optional[np.ndarray] = None, nvalue: int = 0) -> np.ndarray:
        buf = np.frombuffer(bytes(in_), np.uint8).copy()
        o = np.zeros(length, np.uint32)
        _check(lib().leco_block_decode(LINEAR_F32, 4, _np_ptr(buf), len(buf), length, _np_ptr(o)), "decodeArray8")
        if out is None:
            return o
        out[:length] = o
        return out

    def randomdecodeArray8(self, in_, l: int, out=None, nvalue: int = 0, length: Optional[int] = None) -> int:
        buf = np.frombuffer(bytes(in_), np.uint8).copy()
        n = length if length is not None else l + 1
        nbytes = int(lib().leco_block_bytes(LINEAR_F32, 4, int(buf[0]), n))  # the image prefix that holds value l
        v = np.zeros(1, np.uint32)
        _check(lib().leco_block_random(LINEAR_F32, 4, _np_ptr(buf), nbytes, n, l, _np_ptr(v)), "randomdecodeArray8")
        return int(v[0])


class Leco_int_poly(_BlockCodec):
    """Mirror of ``Codecset::Leco_int_poly<T, 2>`` (poly_fix_integer_template.h:15-292)."""
    CODEC = POLY2


# ---------------------------------------------------------------------------
# Container files and the reference's per-block byte strings.
# ---------------------------------------------------------------------------

class ContainerInfo(ctypes.Structure):
    _fields_ = [("codec", ctypes.c_int), ("dtype", ctypes.c_int), ("block_size", ctypes.c_uint32),
                ("n", ctypes.c_uint64), ("nunits", ctypes.c_uint64), ("payload_bytes", ctypes.c_uint64),
                ("has_starts", ctypes.c_int)]


def container_write(path: str, codec: int, dtype: int, block_size: int, n: int, payload: np.ndarray,
                    offsets: np.ndarray, starts: Optional[np.ndarray] = None) -> None:
    """Writes a column (host arrays) to a container file."""
    payload = np.ascontiguousarray(payload, np.uint8)
    offsets = np.ascontiguousarray(offsets, np.uint64)
    info = ContainerInfo(codec, dtype, block_size, n, len(offsets) - 1, int(offsets[-1]), int(starts is not None))
    st = np.ascontiguousarray(starts, np.uint64) if starts is not None else None
    _check(lib().leco_container_write(os.fsencode(path), ctypes.byref(info), _np_ptr(payload), _np_ptr(offsets),
                                      _np_ptr(st) if st is not None else None), "leco_container_write")


def container_info(path: str) -> dict:
    info = ContainerInfo()
    _check(lib().leco_container_info_read(os.fsencode(path), ctypes.byref(info)), "leco_container_info_read")
    return {f: getattr(info, f) for f, _ in ContainerInfo._fields_}


def container_read(path: str):
    """(info dict, payload uint8, offsets uint64, starts uint64 or None) of a
    container file, checked (header, offsets, checksum, block headers)."""
    info = container_info(path)
    pay = np.zeros(info["payload_bytes"], np.uint8)
    off = np.zeros(info["nunits"] + 1, np.uint64)
    st = np.zeros(info["nunits"], np.uint64) if info["has_starts"] else None
    _check(lib().leco_container_read(os.fsencode(path), _np_ptr(pay), len(pay), _np_ptr(off),
                                     _np_ptr(st) if st is not None else None), "leco_container_read")
    return info, pay, off, st


def import_blocks(blocks) -> tuple:
    """The reference drivers' per-block byte strings -> (payload, offsets)."""
    blocks = [bytes(b) for b in blocks]
    bufs = [np.frombuffer(b, np.uint8) for b in blocks]
    ptrs = (ctypes.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
    sizes = np.array([len(b) for b in blocks], np.uint64)
    pay = np.zeros(int(sizes.sum()), np.uint8)
    off = np.zeros(len(blocks) + 1, np.uint64)
    _check(lib().leco_import_blocks(ptrs, _np_ptr(sizes), len(blocks), _np_ptr(pay), len(pay), _np_ptr(off)),
           "leco_import_blocks")
    return pay, off


def export_blocks(payload: np.ndarray, offsets: np.ndarray) -> list:
    """(payload, offsets) -> the per-block byte strings, as the reference's
    encodeArray8_int returned them."""
    payload = np.ascontiguousarray(payload, np.uint8)
    offsets = np.ascontiguousarray(offsets, np.uint64)
    nb = len(offsets) - 1
    sizes = np.zeros(nb, np.uint64)
    _check(lib().leco_export_blocks(_np_ptr(payload), _np_ptr(offsets), nb, None, _np_ptr(sizes)), "leco_export_blocks")
    bufs = [np.zeros(int(z), np.uint8) for z in sizes]
    ptrs = (ctypes.c_void_p * nb)(*[b.ctypes.data for b in bufs])
    _check(lib().leco_export_blocks(_np_ptr(payload), _np_ptr(offsets), nb, ptrs, _np_ptr(sizes)), "leco_export_blocks")
    return [b.tobytes() for b in bufs]


# ---------------------------------------------------------------------------
# Device-resident columns.
# ---------------------------------------------------------------------------

def _torch():
    import torch  # plumbing only: device allocations and stream handles
    return torch


def _stream_ptr(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return _P(s.cuda_stream)


def _tptr(t):
    return _P(t.data_ptr()) if t is not None else None


_TORCH_INT = {4: "int32", 8: "int64"}


@dataclass
class Column:
    """An encoded column in device memory.

    ``payload`` holds the reference block images back to back (plus
    PAYLOAD_SLACK bytes), ``offsets[b]`` the byte offset of block b
    (``offsets[nblocks]`` = compressed bytes), ``dir`` the 32-byte per-block
    directory used by random access.
    """
    codec: int
    dtype: int
    n: int
    block_size: int
    payload: object
    offsets: object
    dir: object = None
    _nbytes: Optional[int] = field(default=None, repr=False)

    @property
    def nblocks(self) -> int:
        return (self.n + self.block_size - 1) // self.block_size

    @property
    def nbytes(self) -> int:
        """Compressed bytes: the sum of the reference block image sizes."""
        if self._nbytes is None:
            self._nbytes = int(self.offsets[-1].item())
        return self._nbytes

    @property
    def ratio(self) -> float:
        return self.nbytes / (self.n * self.dtype)

    def decode(self, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty(self.n, dtype=getattr(torch, _TORCH_INT[self.dtype]), device=self.payload.device)
        _check(lib().leco_decode(self.codec, self.dtype, _tptr(self.payload), _tptr(self.offsets), self.n, self.block_size,
                                 _tptr(out), _stream_ptr(stream)), "leco_decode")
        return out

    def decode_range(self, first: int, count: int, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty(count, dtype=getattr(torch, _TORCH_INT[self.dtype]), device=self.payload.device)
        _check(lib().leco_decode_range(self.codec, self.dtype, _tptr(self.payload), _tptr(self.offsets), self.n,
                                       self.block_size, first, count, _tptr(out), _stream_ptr(stream)), "leco_decode_range")
        return out

    def gather(self, idx, out=None, stream=None, use_dir: bool = True):
        torch = _torch()
        if out is None:
            out = torch.empty(idx.numel(), dtype=getattr(torch, _TORCH_INT[self.dtype]), device=self.payload.device)
        _check(lib().leco_gather(self.codec, self.dtype, _tptr(self.payload), _tptr(self.offsets),
                                 _tptr(self.dir) if use_dir else None, self.n, self.block_size, _tptr(idx), idx.numel(),
                                 _tptr(out), _stream_ptr(stream)), "leco_gather")
        return out

    def sum(self, out=None, stream=None) -> int:
        torch = _torch()
        if out is None:
            out = torch.empty(1, dtype=torch.int64, device=self.payload.device)
        _check(lib().leco_sum(self.codec, self.dtype, _tptr(self.payload), _tptr(self.offsets), self.n, self.block_size,
                              _tptr(out), None, _stream_ptr(stream)), "leco_sum")
        return int(out.item()) & 0xFFFFFFFFFFFFFFFF

    # -- predicate pushdown (Leco_int / FOR_int filter_range, filter_range_close) --
    def zonemap(self, stream=None):
        """(min, max) of every block's decoded values, as int64 tensors holding
        the uint64 bit patterns."""
        torch = _torch()
        zmin = torch.empty(self.nblocks, dtype=torch.int64, device=self.payload.device)
        zmax = torch.empty_like(zmin)
        _check(lib().leco_zonemap(self.codec, self.dtype, _tptr(self.payload), _tptr(self.offsets), self.n,
                                  self.block_size, _tptr(zmin), _tptr(zmax), _stream_ptr(stream)), "leco_zonemap")
        return zmin, zmax

    def _filter_buffers(self, out, out_cap, ws):
        torch = _torch()
        dev = self.payload.device
        if out is None:
            out_cap = self.n + self.nblocks if out_cap is None else out_cap
            out = torch.empty(max(out_cap, 1), dtype=torch.int32, device=dev)
        elif out_cap is None:
            out_cap = out.numel()
        need = int(lib().leco_filter_workspace_bytes(self.n, self.block_size))
        if ws is None or ws.numel() < need:
            ws = torch.empty(need, dtype=torch.uint8, device=dev)
        count = torch.empty(1, dtype=torch.int64, device=dev)
        return out, out_cap, ws, count

    def filter_range(self, filt: int, zone_max=None, zone_min=None, out=None, out_cap=None, ws=None, stream=None,
                     sync: bool = True):
        """Indices (int32 tensor holding uint32) of the values above `filt`;
        returns (indices, count).  sync=False returns the device count tensor
        and the full output buffer without waiting."""
        out, out_cap, ws, count = self._filter_buffers(out, out_cap, ws)
        _check(lib().leco_filter_range(self.codec, self.dtype, _tptr(self.payload), _tptr(self.offsets), self.n,
                                       self.block_size, int(filt) & 0xFFFFFFFFFFFFFFFF, _tptr(zone_min),
                                       _tptr(zone_max), _tptr(out),
                                       out_cap, _tptr(count), _tptr(ws), ws.numel(), _stream_ptr(stream)),
               "leco_filter_range")
        if not sync:
            return out, count
        c = int(count.item())
        return out[:min(c, out_cap)], c

    def filter_range_close(self, f1: int, f2: int, base: int, zone_min=None, out=None, out_cap=None, ws=None,
                           stream=None, sync: bool = True):
        """Close-range filter (windows (f1 + p*base, f2 + p*base) for LeCo,
        residues f1 < v % base < f2 for FOR); returns (indices, count)."""
        out, out_cap, ws, count = self._filter_buffers(out, out_cap, ws)
        _check(lib().leco_filter_range_close(self.codec, self.dtype, _tptr(self.payload), _tptr(self.offsets), self.n,
                                             self.block_size, int(f1) & 0xFFFFFFFFFFFFFFFF, int(f2) & 0xFFFFFFFFFFFFFFFF,
                                             base, _tptr(zone_min), _tptr(out), out_cap, _tptr(count), _tptr(ws),
                                             ws.numel(), _stream_ptr(stream)), "leco_filter_range_close")
        if not sync:
            return out, count
        c = int(count.item())
        _check(lib().leco_check(_stream_ptr(stream)), "leco_filter_range_close")
        return out[:min(c, out_cap)], c

    def build_directory(self, stream=None):
        torch = _torch()
        if self.dir is None:
            self.dir = torch.empty(self.nblocks * 32, dtype=torch.uint8, device=self.payload.device)
        _check(lib().leco_build_directory(self.codec, self.dtype, _tptr(self.payload), _tptr(self.offsets), self.n,
                                          self.block_size, _tptr(self.dir), _stream_ptr(stream)), "leco_build_directory")
        return self.dir

    def compact(self):
        """Moves the payload into an exactly sized buffer (encode allocates the
        worst case); returns self."""
        torch = _torch()
        n = self.nbytes
        buf = torch.zeros(n + PAYLOAD_SLACK, dtype=torch.uint8, device=self.payload.device)
        buf[:n].copy_(self.payload[:n])
        self.payload = buf
        if self.dir is not None:  # the directory holds bit addresses, not pointers: still valid
            pass
        return self

    def to_host(self):
        """(payload bytes as uint8 numpy, offsets as uint64 numpy)."""
        off = self.offsets.cpu().numpy().view(np.uint64)
        pay = self.payload[: int(off[-1])].cpu().numpy()
        return pay, off

    def save(self, path: str, stream=None) -> None:
        """Writes the column to a container file (leco_container_save_device)."""
        info = ContainerInfo(self.codec, self.dtype, self.block_size, self.n, self.nblocks, self.nbytes, 0)
        _check(lib().leco_container_save_device(os.fsencode(path), ctypes.byref(info), _tptr(self.payload),
                                                _tptr(self.offsets), None, _stream_ptr(stream)), "leco_container_save_device")

    @classmethod
    def load(cls, path: str, device="cuda", stream=None) -> "Column":
        """A column read from a container file into device memory (checked
        before it reaches a kernel), with its random-access directory."""
        torch = _torch()
        info = container_info(path)
        if info["codec"] == VARLEN:
            raise LecoError(-1, "a variable-length container: use VarlenColumn.load")
        pay = torch.empty(info["payload_bytes"] + PAYLOAD_SLACK, dtype=torch.uint8, device=device)
        off = torch.empty(info["nunits"] + 1, dtype=torch.int64, device=device)
        _check(lib().leco_container_load_device(os.fsencode(path), _tptr(pay), pay.numel(), _tptr(off), None,
                                                _stream_ptr(stream)), "leco_container_load_device")
        col = cls(info["codec"], info["dtype"], info["n"], info["block_size"], pay, off)
        col.build_directory()
        return col

    @classmethod
    def from_host(cls, codec: int, dtype: int, n: int, block_size: int, payload: np.ndarray, offsets: np.ndarray,
                  device="cuda", validate: bool = True) -> "Column":
        """Imports reference block images (e.g. from the reference encoder)."""
        torch = _torch()
        payload = np.ascontiguousarray(payload, np.uint8)
        offsets = np.ascontiguousarray(offsets, np.uint64)
        if validate:
            bad = np.zeros(1, np.uint64)
            _check(lib().leco_validate_host(codec, dtype, _np_ptr(payload), len(payload), _np_ptr(offsets), n, block_size,
                                            _np_ptr(bad)), "leco_validate_host")
        buf = np.zeros(len(payload) + PAYLOAD_SLACK, np.uint8)
        buf[: len(payload)] = payload
        col = cls(codec, dtype, n, block_size, torch.from_numpy(buf).to(device),
                  torch.from_numpy(offsets.view(np.int64)).to(device))
        col.build_directory()
        return col


def check(stream=None) -> None:
    """Raises if a kernel set the device error word (bad index, header, timeout)."""
    _check(lib().leco_check(_stream_ptr(stream)), "leco_check")


def encode(values, codec: int = LINEAR, block_size: int = 4096, fit_mode: int = FIT_REFERENCE, stream=None,
           with_dir: bool = True, workspace=None, payload=None) -> Column:
    """Encodes a 1-D CUDA tensor of 32/64-bit integers (viewed as unsigned)."""
    torch = _torch()
    if not values.is_cuda:
        raise ValueError("values must be a CUDA tensor")
    s = values.element_size()
    n = values.numel()
    L = lib()
    nb = L.leco_num_blocks(n, block_size)
    cap = L.leco_max_payload_bytes(codec, s, n, block_size)
    wsb = L.leco_encode_workspace_bytes(codec, s, n, block_size, fit_mode)
    dev = values.device
    if payload is None or payload.numel() < cap:
        payload = torch.empty(cap, dtype=torch.uint8, device=dev)
    offsets = torch.empty(nb + 1, dtype=torch.int64, device=dev)
    d = torch.empty(nb * 32, dtype=torch.uint8, device=dev) if with_dir else None
    if workspace is None or workspace.numel() < wsb:
        workspace = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
    _check(L.leco_encode(codec, s, _tptr(values), n, block_size, fit_mode, _tptr(payload), cap, _tptr(offsets), _tptr(d),
                         _tptr(workspace), wsb, _stream_ptr(stream)), "leco_encode")
    return Column(codec, s, n, block_size, payload, offsets, d)


def version() -> str:
    return lib().leco_version().decode()


# ---------------------------------------------------------------------------
# Batch engine: many columns, one persistent launch per pass.
# ---------------------------------------------------------------------------

class ColumnDesc(ctypes.Structure):
    """``leco_column_desc`` of include/leco.h."""
    _fields_ = [("codec", ctypes.c_int32), ("dtype", ctypes.c_int32), ("block_size", ctypes.c_uint32),
                ("group_threads", ctypes.c_uint16), ("unroll", ctypes.c_uint16), ("n", ctypes.c_uint64),
                ("d_values", _P), ("d_out", _P),
                ("d_payload", _P), ("payload_cap", ctypes.c_uint64), ("d_offsets", _P), ("d_dir", _P)]


class Batch:
    """Columns encoded/decoded together by the persistent batch kernels.

    ``columns``: list of (values CUDA tensor, codec, block_size) or
    (values, codec, block_size, group_threads, unroll) -- the autotune table's
    three parameters; 0 (or absent) takes the engine's defaults.  Payload,
    offsets, directory and decode-output tensors are allocated here; the C
    side keeps only raw pointers, so this object owns them.
    """

    def __init__(self, columns, fit_mode: int = FIT_REFERENCE, decode_out: bool = True):
        torch = _torch()
        L = lib()
        self.fit_mode = fit_mode
        self.values, self.cols = [], []
        descs = (ColumnDesc * len(columns))()
        for i, spec in enumerate(columns):
            v, codec, bs = spec[:3]
            group, unroll = (int(spec[3]), int(spec[4])) if len(spec) > 3 else (0, 0)
            s, n = v.element_size(), v.numel()
            nb = L.leco_num_blocks(n, bs)
            cap = L.leco_max_payload_bytes(codec, s, n, bs)
            pay = torch.empty(cap, dtype=torch.uint8, device=v.device)
            off = torch.empty(nb + 1, dtype=torch.int64, device=v.device)
            d = torch.empty(nb * 32, dtype=torch.uint8, device=v.device)
            out = torch.empty_like(v) if decode_out else None
            col = Column(codec, s, n, bs, pay, off, d)
            col.out = out
            self.values.append(v)
            self.cols.append(col)
            descs[i] = ColumnDesc(codec, s, bs, group, unroll, n, v.data_ptr(), out.data_ptr() if out is not None else None,
                                  pay.data_ptr(), cap, off.data_ptr(), d.data_ptr())
        self._descs = descs
        h = _P()
        _check(L.leco_batch_create(descs, len(columns), fit_mode, ctypes.byref(h)), "leco_batch_create")
        self._h = h

    @property
    def total_blocks(self) -> int:
        return lib().leco_batch_total_blocks(self._h)

    def encode(self, stream=None):
        _check(lib().leco_batch_encode(self._h, _stream_ptr(stream)), "leco_batch_encode")

    def decode(self, stream=None):
        _check(lib().leco_batch_decode(self._h, _stream_ptr(stream)), "leco_batch_decode")

    def run_graph(self, passes: int = 3, stream=None):
        """passes: 1 encode, 2 decode, 3 both -- captured once, replayed after."""
        _check(lib().leco_batch_run_graph(self._h, passes, _stream_ptr(stream)), "leco_batch_run_graph")

    def encode_per_column(self, stream=None):
        _check(lib().leco_batch_encode_per_column(self._h, _stream_ptr(stream)), "leco_batch_encode_per_column")

    def decode_per_column(self, stream=None):
        _check(lib().leco_batch_decode_per_column(self._h, _stream_ptr(stream)), "leco_batch_decode_per_column")

    def close(self):
        if getattr(self, "_h", None):
            lib().leco_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Serving loop: continuous batching of lookups and range scans.
# ---------------------------------------------------------------------------

REQ_LOOKUP, REQ_RANGE = 0, 1


class Request(ctypes.Structure):
    """``leco_request`` of include/leco.h."""
    _fields_ = [("column", ctypes.c_uint32), ("kind", ctypes.c_uint32), ("count", ctypes.c_uint64),
                ("h_idx", _P), ("first", ctypes.c_uint64), ("h_out", _P)]


class ServerOptions(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_uint32), ("max_requests_per_batch", ctypes.c_uint32),
                ("max_items_per_batch", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("hbm_budget_bytes", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("lookups", ctypes.c_uint64), ("scanned_values", ctypes.c_uint64),
                ("batches", ctypes.c_uint64), ("max_requests_in_batch", ctypes.c_uint64), ("arena_bytes", ctypes.c_uint64),
                ("p50_us", ctypes.c_double), ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double),
                ("max_us", ctypes.c_double)]


class Server:
    """A request loop over resident encoded ``Column`` objects.

    ``submit`` takes pinned host buffers (torch ``pin_memory=True`` tensors):
    ``idx`` (int64 indices) for a lookup or ``first`` for a range scan, and
    ``out`` for the results.  The buffers must stay alive until ``wait``
    returns for that request."""

    def __init__(self, columns, slots: int = 4, max_requests_per_batch: int = 1024, hbm_budget_bytes: int = 0,
                 max_items_per_batch: int = 0):
        L = lib()
        self.columns = list(columns)
        descs = (ColumnDesc * len(self.columns))()
        for i, c in enumerate(self.columns):
            if c.dir is None:
                c.build_directory()
            descs[i] = ColumnDesc(c.codec, c.dtype, c.block_size, 0, 0, c.n, None, None, c.payload.data_ptr(),
                                  c.payload.numel(), c.offsets.data_ptr(), c.dir.data_ptr())
        self.options = dict(slots=slots, max_requests_per_batch=max_requests_per_batch,
                            hbm_budget_bytes=hbm_budget_bytes, max_items_per_batch=max_items_per_batch)
        opt = ServerOptions(slots, max_requests_per_batch, max_items_per_batch, 0, hbm_budget_bytes)
        h = _P()
        _check(L.leco_server_create(descs, len(self.columns), ctypes.byref(opt), ctypes.byref(h)), "leco_server_create")
        self._h = h

    def submit(self, column: int, out, idx=None, first: int = 0, count: int | None = None) -> int:
        if idx is not None:
            r = Request(column, REQ_LOOKUP, idx.numel(), idx.data_ptr(), 0, out.data_ptr())
        else:
            r = Request(column, REQ_RANGE, count if count is not None else out.numel(), None, first, out.data_ptr())
        rid = ctypes.c_uint64()
        _check(lib().leco_server_submit(self._h, ctypes.byref(r), ctypes.byref(rid)), "leco_server_submit")
        return rid.value

    def wait(self, rid: int) -> float:
        lat = ctypes.c_double()
        _check(lib().leco_server_wait(self._h, rid, ctypes.byref(lat)), "leco_server_wait")
        return lat.value

    def drain(self):
        _check(lib().leco_server_drain(self._h), "leco_server_drain")

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().leco_server_get_stats(self._h, ctypes.byref(st)), "leco_server_get_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def reset_stats(self):
        _check(lib().leco_server_reset_stats(self._h), "leco_server_reset_stats")

    def checkpoint(self, directory: str) -> None:
        """Saves the resident columns (one container file each) and the server
        options (manifest.json) after draining the requests in flight."""
        import json

        self.drain()
        os.makedirs(directory, exist_ok=True)
        names = []
        for i, c in enumerate(self.columns):
            name = f"column_{i:05d}.leco"
            c.save(os.path.join(directory, name))
            names.append(name)
        tmp = os.path.join(directory, "manifest.json.tmp")
        with open(tmp, "w") as f:
            json.dump({"format": "leco-server-checkpoint-1", "columns": names, "options": self.options}, f)
        os.replace(tmp, os.path.join(directory, "manifest.json"))

    @classmethod
    def resume(cls, directory: str, device="cuda") -> "Server":
        """A server over the columns of a checkpoint, with its options."""
        import json

        with open(os.path.join(directory, "manifest.json")) as f:
            m = json.load(f)
        if m.get("format") != "leco-server-checkpoint-1":
            raise LecoError(-3, f"{directory}: not a server checkpoint")
        cols = [Column.load(os.path.join(directory, name), device=device) for name in m["columns"]]
        return cls(cols, **m["options"])

    def close(self):
        if getattr(self, "_h", None):
            lib().leco_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Variable-length segments.
# ---------------------------------------------------------------------------

def varlen_partition(values: np.ndarray, coarse_blocks: int, delta: int, threads: int = 0) -> np.ndarray:
    """Segment starts (uint64) of a uint64 column, computed on the host cores."""
    values = np.ascontiguousarray(values, np.uint64)
    out = np.zeros(len(values), np.uint64)
    ns = ctypes.c_uint64()
    _check(lib().leco_varlen_partition(_np_ptr(values), len(values), coarse_blocks, delta, _np_ptr(out), len(out),
                                       ctypes.byref(ns), threads), "leco_varlen_partition")
    return out[: ns.value].copy()


def varlen_partition_device(values, coarse_blocks: int, delta: int, ws=None, stream=None):
    """Segment starts (int64 CUDA tensor holding uint64) of a uint64 column
    already on the device (int64 tensor), computed on the GPU."""
    torch = _torch()
    n = values.numel()
    need = int(lib().leco_varlen_partition_workspace_bytes(n, coarse_blocks))
    if ws is None or ws.numel() < need:
        ws = torch.empty(need, dtype=torch.uint8, device=values.device)
    starts = torch.empty(n, dtype=torch.int64, device=values.device)
    nseg = torch.zeros(1, dtype=torch.int64, device=values.device)
    _check(lib().leco_varlen_partition_device(_tptr(values), n, coarse_blocks, delta, _tptr(starts), n, _tptr(nseg),
                                              _tptr(ws), ws.numel(), _stream_ptr(stream)), "leco_varlen_partition_device")
    k = int(nseg.item())
    _check(lib().leco_check(_stream_ptr(stream)), "leco_varlen_partition_device")
    return starts[:k]


@dataclass
class VarlenColumn:
    n: int
    starts: object   # int64 CUDA tensor [nseg]
    payload: object  # uint8 CUDA tensor
    offsets: object  # int64 CUDA tensor [nseg + 1]

    @property
    def nseg(self) -> int:
        return self.starts.numel()

    @property
    def nbytes(self) -> int:
        return int(self.offsets[-1].item())

    def decode(self, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty(self.n, dtype=torch.int64, device=self.payload.device)
        _check(lib().leco_varlen_decode(_tptr(self.payload), _tptr(self.offsets), _tptr(self.starts), self.nseg, self.n,
                                        _tptr(out), _stream_ptr(stream)), "leco_varlen_decode")
        return out

    def gather(self, idx, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty(idx.numel(), dtype=torch.int64, device=self.payload.device)
        _check(lib().leco_varlen_gather(_tptr(self.payload), _tptr(self.offsets), _tptr(self.starts), self.nseg, self.n,
                                        _tptr(idx), idx.numel(), _tptr(out), _stream_ptr(stream)), "leco_varlen_gather")
        return out

    def sum(self, stream=None) -> int:
        torch = _torch()
        out = torch.empty(1, dtype=torch.int64, device=self.payload.device)
        _check(lib().leco_varlen_sum(_tptr(self.payload), _tptr(self.offsets), _tptr(self.starts), self.nseg, self.n,
                                     _tptr(out), _stream_ptr(stream)), "leco_varlen_sum")
        return int(out.item()) & 0xFFFFFFFFFFFFFFFF

    def to_host(self):
        off = self.offsets.cpu().numpy().view(np.uint64)
        return self.payload[: int(off[-1])].cpu().numpy(), off, self.starts.cpu().numpy().view(np.uint64)

    def save(self, path: str, stream=None) -> None:
        info = ContainerInfo(VARLEN, 8, 0, self.n, self.nseg, self.nbytes, 1)
        _check(lib().leco_container_save_device(os.fsencode(path), ctypes.byref(info), _tptr(self.payload),
                                                _tptr(self.offsets), _tptr(self.starts), _stream_ptr(stream)),
               "leco_container_save_device")

    @classmethod
    def load(cls, path: str, device="cuda", stream=None) -> "VarlenColumn":
        torch = _torch()
        info = container_info(path)
        if info["codec"] != VARLEN:
            raise LecoError(-1, "a fixed-block container: use Column.load")
        pay = torch.empty(info["payload_bytes"] + PAYLOAD_SLACK, dtype=torch.uint8, device=device)
        off = torch.empty(info["nunits"] + 1, dtype=torch.int64, device=device)
        st = torch.empty(info["nunits"], dtype=torch.int64, device=device)
        _check(lib().leco_container_load_device(os.fsencode(path), _tptr(pay), pay.numel(), _tptr(off), _tptr(st),
                                                _stream_ptr(stream)), "leco_container_load_device")
        return cls(info["n"], st, pay, off)


def varlen_encode(values, starts, fit_mode: int = FIT_REFERENCE, stream=None, max_segment_len: int = 0) -> VarlenColumn:
    """Encodes a uint64 CUDA tensor (int64 view) with the given segment starts
    (host numpy array, or a CUDA tensor together with max_segment_len)."""
    torch = _torch()
    L = lib()
    n = values.numel()
    if not hasattr(starts, "is_cuda"):
        sh = np.ascontiguousarray(starts, np.uint64)
        max_segment_len = int(np.max(np.diff(np.append(sh, np.uint64(n))))) if len(sh) else 0
        st = torch.from_numpy(sh.view(np.int64))
    else:
        st = starts
    st = st.to(values.device)
    ns = st.numel()
    cap = L.leco_varlen_max_payload_bytes(n, ns)
    pay = torch.empty(cap, dtype=torch.uint8, device=values.device)
    off = torch.empty(ns + 1, dtype=torch.int64, device=values.device)
    wsb = L.leco_varlen_workspace_bytes(ns)
    ws = torch.empty(wsb, dtype=torch.uint8, device=values.device)
    _check(L.leco_varlen_encode(_tptr(values), n, _tptr(st), ns, max_segment_len, fit_mode, _tptr(pay), cap, _tptr(off),
                                _tptr(ws), wsb, _stream_ptr(stream)), "leco_varlen_encode")
    col = VarlenColumn(n, st, pay, off)
    col.max_segment_len = max_segment_len
    return col
