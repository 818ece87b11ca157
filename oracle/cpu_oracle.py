"""ctypes wrapper of ``oracle/cpu_decoder.c``: TEST INFRASTRUCTURE ONLY.

Decodes a whole BAM file on the host cores (zlib inflate per member in
parallel, the record chain, the columns and tags) with the semantics of
``oracle/bam_oracle.py``.  Used by tests as the oracle for inputs too large for
the Python oracle, and by ``bench.py`` as the timed CPU baseline.
"""

from __future__ import annotations

import ctypes
import os
import time
from ctypes import POINTER, c_char_p, c_int, c_int64, c_void_p
from dataclasses import dataclass, field

import numpy as np

from oracle import build_oracle
from oracle.bam_oracle import read_header

_lib = None
_P = c_void_p


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.build()
        _lib = ctypes.CDLL(str(path))
        _lib.orc_scan_file.restype = c_int64
        _lib.orc_scan_file.argtypes = [_P, c_int64, _P, _P, _P, _P, c_int64, c_int]
        _lib.orc_inflate.restype = c_int
        _lib.orc_inflate.argtypes = [_P, _P, _P, _P, _P, c_int64, _P, c_int, c_int]
        _lib.orc_record_chain.restype = c_int64
        _lib.orc_record_chain.argtypes = [_P, c_int64, c_int64, c_int, _P, c_int64, POINTER(c_int64)]
        _lib.orc_decode.restype = c_int
        _lib.orc_decode.argtypes = [_P, _P, c_int64, c_int] + [_P] * 12 + [c_int, c_char_p] + [_P] * 5
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data


@dataclass
class Decoded:
    data: np.ndarray  # inflated records area (header skipped)
    offset: np.ndarray
    columns: dict
    name_hash: np.ndarray
    tags: dict = field(default_factory=dict)  # name -> (type, voff, vlen, value, hash)
    seconds: dict = field(default_factory=dict)
    n_members: int = 0
    inflated_bytes: int = 0
    compressed_bytes: int = 0


FIELDS = ("ref", "pos", "end", "mapq", "flag", "nref", "npos", "tlen", "l_seq", "clip_left", "clip_right")
_DT = dict(ref=np.int32, pos=np.int32, end=np.int32, mapq=np.uint8, flag=np.uint16, nref=np.int32, npos=np.int32,
           tlen=np.int32, l_seq=np.int32, clip_left=np.uint16, clip_right=np.uint16)


def _buf(ws: dict | None, name: str, n: int, dtype, shape=None) -> np.ndarray:
    """An array of ``n`` elements, taken from (and kept in) the workspace ``ws`` when one is given, so that
    repeated decodes of the same file do not fault in fresh pages every time."""
    shape = shape or (n,)
    size = int(np.prod(shape))
    if ws is None:
        return np.empty(shape, dtype)
    a = ws.get(name)
    if a is None or a.dtype != np.dtype(dtype) or a.size < size:
        a = np.empty(size, dtype)
        ws[name] = a
    return a[:size].reshape(shape)


def inflate_file(raw: bytes | np.ndarray, n_threads: int | None = None, check_crc: bool = True,
                 prefix_bytes: int | None = None, ws: dict | None = None):
    """``(inflated uint8 array, n_members, compressed bytes used)`` of a whole BGZF file, or of the
    members within its first ``prefix_bytes`` bytes."""
    L = lib()
    f = np.frombuffer(raw, np.uint8) if not isinstance(raw, np.ndarray) else raw
    n = f.size if prefix_bytes is None else min(f.size, int(prefix_bytes))
    cap = n // 26 + 2
    off, bs, isz, oo = (_buf(ws, k, cap, np.int64) for k in ("m_off", "m_bs", "m_isz", "m_oo"))
    m = L.orc_scan_file(_p(f), n, _p(off), _p(bs), _p(isz), _p(oo), cap, int(prefix_bytes is not None))
    if m < 0:
        raise ValueError(f"BGZF scan failed (status {-m})")
    total = int(oo[m - 1] + isz[m - 1]) if m else 0
    used = int(off[m - 1] + bs[m - 1]) if m else 0
    out = _buf(ws, "inflated", max(total, 1), np.uint8)
    st = L.orc_inflate(_p(f), _p(off), _p(bs), _p(isz), _p(oo), m, _p(out), n_threads or os.cpu_count(),
                       int(check_crc))
    if st:
        raise ValueError(f"inflate failed (status {st})")
    return out[:total], int(m), used


def decode_file(raw: bytes, n_threads: int | None = None, tags=("CB", "UB", "GN"), check_crc: bool = True,
                prefix_bytes: int | None = None, ws: dict | None = None) -> Decoded:
    """All records of a BAM file (or of its first ``prefix_bytes`` compressed bytes), on ``n_threads`` threads.
    ``ws``: a dict that keeps the output arrays between calls (the results then share its memory)."""
    L = lib()
    nt = n_threads or os.cpu_count()
    t0 = time.perf_counter()
    data, m, used = inflate_file(raw, nt, check_crc, prefix_bytes, ws)
    t1 = time.perf_counter()
    _, names, _, skip = read_header(bytes(raw[: min(len(raw), 1 << 20)]) if len(raw) > (1 << 20) else raw)
    data = data[skip:]  # offsets are relative to the records area, as in cubam's batches
    cap = max(data.size // 37 + 2, 1)
    off = _buf(ws, "offset", cap, np.int64)
    tail = c_int64(0)
    nrec = L.orc_record_chain(_p(data), data.size, 0, len(names), _p(off), cap, ctypes.byref(tail))
    if nrec < 0:
        raise ValueError("record chain overflow")
    if tail.value != data.size and prefix_bytes is None:
        raise ValueError("truncated BAM file (incomplete record at the end)")
    off = off[:nrec]
    t2 = time.perf_counter()
    cols = {k: _buf(ws, "col_" + k, nrec, t) for k, t in _DT.items()}
    nh = _buf(ws, "name_hash", nrec, np.uint64)
    k = len(tags)
    ty = _buf(ws, "tag_type", 0, np.uint8, (k, nrec))
    vo = _buf(ws, "tag_offset", 0, np.int64, (k, nrec))
    vl = _buf(ws, "tag_length", 0, np.int32, (k, nrec))
    iv = _buf(ws, "tag_value", 0, np.int64, (k, nrec))
    th = _buf(ws, "tag_hash", 0, np.uint64, (k, nrec))
    L.orc_decode(_p(data), _p(off), nrec, nt, *(_p(cols[f]) for f in FIELDS), _p(nh), k, "".join(tags).encode(),
                 _p(ty), _p(vo), _p(vl), _p(iv), _p(th))
    t3 = time.perf_counter()
    d = Decoded(data, off, cols, nh, n_members=m, inflated_bytes=int(data.size), compressed_bytes=used)
    for q, t in enumerate(tags):
        d.tags[t] = (ty[q], vo[q], vl[q], iv[q], th[q])
    d.seconds = {"inflate": t1 - t0, "chain": t2 - t1, "decode": t3 - t2, "total": t3 - t0}
    return d


def decode_prefix(raw, prefix_bytes: int, n_threads: int | None = None, tags=("CB", "UB", "GN"),
                  ws: dict | None = None) -> Decoded:
    """The members within the first ``prefix_bytes`` bytes of a BAM file (a bounded CPU sample)."""
    return decode_file(raw, n_threads, tags, True, prefix_bytes, ws)
