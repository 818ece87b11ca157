"""ctypes binding of the native library (``include/cubam_b200.h``).

The library is loaded from ``cubam_b200/_lib/libcubam_b200.so``.  There is no
fallback: when it is missing, importing this module raises, and every reader
call fails loudly.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_int, c_int32, c_int64, c_size_t, c_void_p
from pathlib import Path

from cubam_b200 import build as _build

LIB_PATH = _build.LIB

# status codes (include/cubam_b200.h)
OK, TRUNCATED, NO_CHAIN, CORRUPT_BLOCK, INFLATE, CRC, TOO_MANY, CAPACITY, CUDA, ARG, TIMEOUT = range(11)
#: launch parameters (cb_set_param / cb_get_param)
(PARAM_CHAIN_TILE, PARAM_INFLATE_FORM, PARAM_DECODE_ROOT, PARAM_COPY_WARPS, PARAM_DECODE_STEPS, PARAM_DECODE_PREFETCH,
 PARAM_SPLIT_MIN_JOBS, PARAM_COPY_UNITS, PARAM_DECODE_PIPELINE) = range(1, 10)


class MemberJob(ctypes.Structure):
    _fields_ = [
        ("in_ptr", c_void_p),
        ("out_off", c_int64),
        ("in_len", ctypes.c_uint32),
        ("isize", ctypes.c_uint32),
        ("crc", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class ScanSummary(ctypes.Structure):
    _fields_ = [
        ("n_members", c_int64),
        ("n_jobs", c_int64),
        ("used", c_int64),
        ("total_out", c_int64),
        ("n_candidates", c_int64),
        ("status", c_int32),
        ("chained", c_int32),
    ]


class InflateSummary(ctypes.Structure):
    _fields_ = [("status", c_int32), ("reserved", c_int32), ("n_bad", c_int64), ("first_bad", c_int64)]


class ChainSummary(ctypes.Structure):
    _fields_ = [
        ("n_records", c_int64),
        ("tail", c_int64),
        ("n_candidates", c_int64),
        ("status", c_int32),
        ("chained", c_int32),
    ]


class DeflateSummary(ctypes.Structure):
    _fields_ = [("total", c_int64), ("n_stored", c_int64), ("status", c_int32), ("reserved", c_int32)]


JOB_BYTES = ctypes.sizeof(MemberJob)

P = c_void_p
I64 = c_int64

_SIGNATURES = {
    "cb_version": (c_char_p, []),
    "cb_last_error": (c_char_p, []),
    "cb_device_sm_count": (c_int, []),
    "cb_set_param": (c_int, [c_int, I64]),
    "cb_get_param": (I64, [c_int]),
    "cb_scan_workspace_bytes": (c_size_t, [I64]),
    "cb_scan_members": (c_int, [P, I64, c_int, I64, P, I64, P, P, c_size_t, P]),
    "cb_scan_members_noalloc": (c_int, [P, I64, c_int, I64, P, I64, P, P]),
    "cb_inflate_workspace_bytes": (c_size_t, []),
    "cb_inflate": (c_int, [P, I64, P, P, c_int, P, P, P, c_size_t, P]),
    "cb_inflate_form": (c_int, [P, I64, P, P, c_int, P, P, P, c_size_t, c_int, P]),
    "cb_inflate_lane_slots": (I64, []),
    "cb_inflate_split_workspace_bytes": (c_size_t, [I64, I64]),
    "cb_inflate_split": (c_int, [P, I64, P, P, c_int, P, P, P, c_size_t, P]),
    "cb_record_chain_workspace_bytes": (c_size_t, [I64]),
    "cb_record_chain": (c_int, [P, I64, c_int32, P, I64, P, P, c_size_t, P]),
    "cb_first_record": (c_int, [P, I64, c_int32, I64, c_int32, P, P]),
    "cb_decode_fixed": (c_int, [P, P, I64] + [P] * 11 + [P]),
    "cb_decode_records": (c_int, [P, P, I64] + [P] * 13 + [P]),
    "cb_find_tags": (c_int, [P, P, I64, c_char_p, c_int32, P, P, P, P, P]),
    "cb_decode_columns": (c_int, [P, P, I64] + [P] * 15 + [c_char_p, c_int32, P, P, P, P, P]),
    "cb_name_hash": (c_int, [P, P, I64, P, P]),
    "cb_hash_spans": (c_int, [P, P, P, I64, P, P]),
    "cb_pack_acgt": (c_int, [P, P, P, I64, P, P, P]),
    "cb_unpack_acgt": (c_int, [P, P, I64, P, P]),
    "cb_aligned_length": (c_int, [P, P, I64, P, P]),
    "cb_blocks": (c_int, [P, P, I64, c_int, c_int, P, P, P, P, P, P]),
    "cb_base_at": (c_int, [P, P, P, P, I64, P, P]),
    "cb_copy_spans": (c_int, [P, P, P, P, P, I64, P]),
    "cb_record_sizes": (c_int, [P, P, I64, P, P]),
    "cb_deflate_workspace_bytes": (c_size_t, [I64]),
    "cb_deflate_spans": (c_int, [P, P, P, I64, c_int, c_int, P, I64, P, P, P, P, P, c_size_t, P]),
    "cb_crc32_spans": (c_int, [P, P, P, I64, P, P]),
    "cb_adler32_spans": (c_int, [P, P, P, I64, P, P]),
}


class BatchFile(ctypes.Structure):
    """cb_batch_file: one file's results in a native batch (device pointers)."""

    _fields_ = [
        ("data", c_void_p), ("data_bytes", c_int64), ("offsets", c_void_p), ("n_records", c_int64),
        ("n_members", c_int64), ("inflated_bytes", c_int64), ("header_bytes", c_int64), ("n_ref", c_int32),
        ("k_tags", c_int32),
        *((name, c_void_p) for name in ("ref", "pos", "end", "mapq", "flag", "nref", "npos", "tlen", "l_seq",
                                        "clip_left", "clip_right", "tag_type", "tag_voff", "tag_vlen", "tag_value")),
    ]


_SIGNATURES.update({
    "cb_batch_create": (c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(c_int64), c_int32, c_char_p, c_int32, c_int, P,
                                ctypes.POINTER(c_void_p)]),
    "cb_batch_run": (c_int, [P, P]),
    "cb_batch_capture": (c_int, [P, P]),
    "cb_batch_check": (c_int, [P, P]),
    "cb_batch_file_info": (c_int, [P, c_int32, ctypes.POINTER(BatchFile)]),
    "cb_batch_total_jobs": (c_int64, [P]),
    "cb_batch_form": (c_int, [P]),
    "cb_batch_destroy": (None, [P]),
})


def _load() -> ctypes.CDLL:
    if not Path(LIB_PATH).exists():
        raise ImportError(
            f"cubam_b200 native library not found at {LIB_PATH}: build it with `python cubam_b200/build.py`"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class NativeError(RuntimeError):
    """A CUDA or argument error reported by the native library."""


def check(rc: int, what: str) -> None:
    if rc == OK:
        return
    if rc == CUDA:
        raise NativeError(f"{what}: CUDA error: {lib.cb_last_error().decode()}")
    raise NativeError(f"{what}: status {rc}")


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)
