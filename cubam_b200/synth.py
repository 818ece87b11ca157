"""Seeded synthetic BAM files with the shapes of the reader benchmarks (``csrc/host/synth.c``).

``write_bam(path, config)`` writes one file; the configurations are the
benchmark workloads:

- ``small``: 100,000 single-end 90 bp records on one 1 Mb reference, CB/UB tags (seed 0);
- ``gex``: 50,000,000 single-end 91 bp records over the 25 human chromosomes, spliced and
  clipped CIGARs, CB/UB/GN/xf/NH (seed 1);
- ``atac``: 100,000,000 records as 50,000,000 pairs of 50 bp mates, CB from 10,000 (seed 2);
- ``uneven``: 64 files of 10,000 to 20,000,000 records, GEX or ATAC at random, zlib levels 1-9,
  2% stored members (seed 3), see :func:`uneven_files`.

``n_records`` overrides the size (tests use small versions of the same shapes).
:func:`write_bam_process` writes the same file from the generator's executable in a
child process, so that the caller maps none of this package's libraries.  The
module imports nothing of the package at load time: a benchmark process that must
stay free of the decoder can load this file on its own.
"""

from __future__ import annotations

import ctypes
import importlib.util
import math
import os
import random
import subprocess
from dataclasses import dataclass, replace
from pathlib import Path

_lib = None
_builder = None


def _build():
    """``build.py`` beside this file, loaded on its own (it imports nothing of the package)."""
    global _builder
    if _builder is None:
        spec = importlib.util.spec_from_file_location("_cubam_b200_build_synth", Path(__file__).with_name("build.py"))
        _builder = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(_builder)
    return _builder


@dataclass(frozen=True)
class Config:
    name: str
    shape: int  # 0 small, 1 gex, 2 atac
    n_records: int
    seed: int
    level: int = 6  # zlib level; -1 = 1..9 at random per member
    stored_frac: float = 0.0
    n_barcodes: int = 1000


CONFIGS = {
    "small": Config("small", 0, 100_000, 0),
    "gex": Config("gex", 1, 50_000_000, 1),
    "atac": Config("atac", 2, 100_000_000, 2, n_barcodes=10_000),
}


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(_build().build_synth()))
        _lib.synth_bam.restype = ctypes.c_int
        _lib.synth_bam.argtypes = [
            ctypes.c_char_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_int, ctypes.c_double,
            ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
            ctypes.POINTER(ctypes.c_int64),
        ]
    return _lib


@dataclass
class Written:
    path: Path
    config: Config
    record_bytes: int
    members: int
    file_bytes: int


def write_bam(path: str | Path, config: Config | str, n_records: int | None = None, n_threads: int | None = None,
              seed: int | None = None) -> Written:
    cfg = CONFIGS[config] if isinstance(config, str) else config
    if n_records is not None:
        cfg = replace(cfg, n_records=int(n_records))
    if seed is not None:
        cfg = replace(cfg, seed=int(seed))
    rb, mb, fb = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    rc = lib().synth_bam(
        str(path).encode(), cfg.shape, cfg.n_records, cfg.seed, cfg.level, cfg.stored_frac, cfg.n_barcodes,
        n_threads or os.cpu_count() or 1, ctypes.byref(rb), ctypes.byref(mb), ctypes.byref(fb),
    )
    if rc:
        raise OSError(f"cannot write {path}")
    return Written(Path(path), cfg, rb.value, mb.value, fb.value)


def write_bam_process(path: str | Path, config: Config | str, n_records: int | None = None,
                      n_threads: int | None = None) -> Written:
    """:func:`write_bam` run by the generator's executable in a child process (same bytes)."""
    cfg = CONFIGS[config] if isinstance(config, str) else config
    if n_records is not None:
        cfg = replace(cfg, n_records=int(n_records))
    exe = _build().build_synth_exe()
    args = [str(exe), str(path), str(cfg.shape), str(cfg.n_records), str(cfg.seed), str(cfg.level),
            repr(float(cfg.stored_frac)), str(cfg.n_barcodes), str(n_threads or os.cpu_count() or 1)]
    res = subprocess.run(args, capture_output=True, text=True)
    if res.returncode:
        raise OSError(f"cannot write {path}: {res.stderr.strip()}")
    rb, mb, fb = (int(x) for x in res.stdout.split())
    return Written(Path(path), cfg, rb, mb, fb)


def uneven_files(scale: float = 1.0, seed: int = 3) -> list[Config]:
    """The 64 files of the uneven-size batch: log-uniform 10k-20M records (times ``scale``), GEX or ATAC."""
    rng = random.Random(seed)
    out = []
    for i in range(64):
        n = int(math.exp(rng.uniform(math.log(10_000), math.log(20_000_000))) * scale)
        shape = rng.choice([1, 2])
        out.append(Config(f"uneven{i}", shape, max(n, 2), seed * 1000 + i, level=-1, stored_frac=0.02,
                          n_barcodes=1000 if shape == 1 else 10_000))
    return out
