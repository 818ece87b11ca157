"""Reading the golden vectors of ``tests/golden/`` (made by ``tests/golden/make_golden.py``)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
TAGS = ("CB", "UB", "GN", "NM", "XS", "RG", "ZB", "xf", "NH", "XA", "Xc", "XC", "Xs", "Xi", "XI", "Xf", "XH", "ZZ", "QQ")


def meta() -> dict:
    return json.loads((GOLDEN / "golden.json").read_text())


def bam_cases():
    """``(bam file name, chunk bytes)`` of every golden BAM case."""
    return [(name, chunk) for name, chunks in sorted(meta()["bam"].items()) for chunk in chunks]


def _split_strings(lens, chars):
    out, k = [], 0
    for ln in lens.tolist():
        out.append(chars[k : k + ln].tobytes())
        k += ln
    return out


def batches(name: str, chunk: int) -> list[dict]:
    """The golden batches of one case, each a dict of arrays (strings as lists of bytes)."""
    g = np.load(GOLDEN / f"golden_{Path(name).stem}_c{chunk}.npz")
    nb = int(g["n_batches"])
    if nb == 0:
        return []
    n = g["n_records"]
    rec_start = np.concatenate([[0], np.cumsum(n)])
    per_rec = [k for k in g.files if g[k].shape[:1] == (int(n.sum()),) and not k.endswith(("_chars",))]
    per_rec = [k for k in per_rec if not k.startswith(("blocks", "base_")) and k not in ("n_records", "data_size")]
    out = []
    cuts = {}
    for key in ("blocks0", "blocks1", "base"):
        cuts[key] = np.concatenate([[0], np.cumsum(g[f"{key}_n"])])
    str_keys = ["names"] + [f"tag_{t}_str" for t in TAGS]
    str_pos = {k: 0 for k in str_keys}
    for b in range(nb):
        s, e = rec_start[b], rec_start[b + 1]
        d = {k: g[k][s:e] for k in per_rec}
        d["data_size"] = int(g["data_size"][b])
        for key in ("blocks0", "blocks1"):
            a, z = cuts[key][b], cuts[key][b + 1]
            for f in ("rec", "start", "end"):
                d[f"{key}_{f}"] = g[f"{key}_{f}"][a:z]
        a, z = cuts["base"][b], cuts["base"][b + 1]
        for f in ("rec", "pos", "at"):
            d[f"base_{f}"] = g[f"base_{f}"][a:z]
        for k in str_keys:
            lens = g[f"{k}_len"][s:e]
            total = int(lens.sum())
            chars = g[f"{k}_chars"][str_pos[k] : str_pos[k] + total]
            str_pos[k] += total
            d[k] = _split_strings(lens, chars)
        out.append(d)
    return out
