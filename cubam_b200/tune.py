"""Launch parameters chosen by measurement, cached per device and workload shape.

cubam launches its kernels with fixed shapes (``src/cubam/_kernels.py:637-641``) and reads with a
fixed chunk policy (``src/cubam/_memory.py:11-23``).  Here the shapes that matter are launch
parameters of the library (``cb_set_param``): the inflate form, the root bits of form 3's lane
decoder, the warps, window and group size of form 3's copy kernel, the decode steps between lane scheduling
rounds, the input prefetch distance, and the tile of the record chain's walk.  :func:`tune` times
candidates on a real batch (a :class:`~cubam_b200.batch.BatchPlan`), one parameter at a time in the
order of their effect (coordinate descent from the current values), keeps the fastest, applies it
to the process and stores it in a JSON cache:

- key: the device name and SM count, plus the workload's shape -- members per launch and mean ISIZE,
  both rounded to a power of two -- so that one measurement serves every batch of the same shape;
- file: ``$CUBAM_B200_TUNE_CACHE``, else ``~/.cache/cubam_b200/tune.json``.

:func:`apply_cached` sets the parameters of a cached shape without timing anything.
"""

from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path

import torch

from cubam_b200 import _lib

#: candidate values per parameter, in the order they are tuned
CANDIDATES = {
    "inflate_form": (_lib.PARAM_INFLATE_FORM, (1, 2, 3)),
    "decode_root": (_lib.PARAM_DECODE_ROOT, (6, 7, 8)),
    "copy_warps": (_lib.PARAM_COPY_WARPS, (6, 12, 24)),
    "copy_units": (_lib.PARAM_COPY_UNITS, (1, 2, 4)),
    "decode_steps": (_lib.PARAM_DECODE_STEPS, (8, 16, 32)),
    "decode_prefetch": (_lib.PARAM_DECODE_PREFETCH, (0, 4, 8)),
    "decode_pipeline": (_lib.PARAM_DECODE_PIPELINE, (0, 2)),
    "chain_tile": (_lib.PARAM_CHAIN_TILE, (0, 16384, 32768)),
}
#: the stage each parameter is timed on (StageEvents names)
STAGE = {"chain_tile": "chained"}
#: form-3 parameters are tuned only when form 3 wins
FORM3 = ("decode_root", "copy_warps", "copy_units", "decode_steps", "decode_prefetch", "decode_pipeline")


def cache_path() -> Path:
    env = os.environ.get("CUBAM_B200_TUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "cubam_b200" / "tune.json"


def _pow2(x: float) -> int:
    return 1 << max(0, int(round(math.log2(max(x, 1.0)))))


def shape_key(n_members: int, total_out: int) -> str:
    """Device name, SM count and the workload shape, rounded to powers of two."""
    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    sms = int(_lib.lib.cb_device_sm_count())
    mean = total_out / max(n_members, 1)
    return f"{dev}|sm{sms}|members~{_pow2(n_members)}|isize~{_pow2(mean)}"


def load_cache(path: Path | None = None) -> dict:
    p = path or cache_path()
    try:
        return json.loads(p.read_text())
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path: Path | None = None) -> None:
    p = path or cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(f".tmp{os.getpid()}")
    tmp.write_text(json.dumps(cache, indent=1, sort_keys=True))
    tmp.replace(p)


def current() -> dict:
    """The process's current value of every tuned parameter."""
    return {name: int(_lib.lib.cb_get_param(key)) for name, (key, _) in CANDIDATES.items()}


def apply(values: dict) -> None:
    """Set the parameters ``values`` (name -> value) for the process."""
    for name, v in values.items():
        key = CANDIDATES[name][0]
        rc = _lib.lib.cb_set_param(key, int(v))
        if rc != _lib.OK:
            raise ValueError(f"{name}={v}: {_lib.lib.cb_last_error().decode()}")


def apply_cached(n_members: int, total_out: int, path: Path | None = None) -> dict | None:
    """The cached parameters of this shape, applied; None when the shape was never tuned."""
    entry = load_cache(path).get(shape_key(n_members, total_out))
    if entry:
        apply(entry["params"])
        return entry["params"]
    return None


def _time(plan, stage: str, reps: int) -> float:
    from cubam_b200.batch import StageEvents

    plan.launch(plan.form)  # one run to set up (and check) before timing
    torch.cuda.synchronize()
    plan.check()
    best = None
    for _ in range(reps):
        ev = StageEvents()
        plan.launch(plan.form, ev)
        torch.cuda.synchronize()
        ms = ev.ms()[stage]
        best = ms if best is None else min(best, ms)
    return best


def tune(plan, reps: int = 2, path: Path | None = None, names=None, use_cache: bool = True) -> dict:
    """Tune the launch parameters on ``plan`` (a BatchPlan), apply and cache the best; returns
    ``{"params": {...}, "ms": {name: {value: milliseconds}}, "seconds": tuning time, "key": ...}``."""
    n_members, total = plan.job_base[-1], plan.total_out
    key = shape_key(n_members, total)
    cache = load_cache(path)
    if use_cache and key in cache:
        apply(cache[key]["params"])
        plan.form = cache[key]["params"]["inflate_form"]
        return cache[key]
    t0 = time.perf_counter()
    best = current()
    best["inflate_form"] = plan.form or best["inflate_form"]
    measured = {}
    for name in names or CANDIDATES:
        if name in FORM3 and best["inflate_form"] != 3:
            continue
        stage = STAGE.get(name, "inflated")
        times = {}
        for v in CANDIDATES[name][1]:
            trial = dict(best, **{name: v})
            apply(trial)
            plan.form = trial["inflate_form"]
            times[v] = _time(plan, stage, reps)
        best[name] = min(times, key=times.get)
        measured[name] = times
        apply(best)
        plan.form = best["inflate_form"]
    entry = {"params": best, "ms": {k: {str(a): b for a, b in v.items()} for k, v in measured.items()},
             "seconds": round(time.perf_counter() - t0, 2), "key": key}
    cache[key] = entry
    save_cache(cache, path)
    return entry
