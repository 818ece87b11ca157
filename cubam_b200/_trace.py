"""NVTX ranges around the stages of a decode, for timeline profilers (Nsight Systems).

Off unless the environment sets ``CUBAM_B200_NVTX`` (to anything but ``0``), so that a decode pays
nothing for it.  The stages are the ones :class:`cubam_b200.batch.StageEvents` times: member scan,
inflate, record chain, record pass; each stage boundary closes one range and opens the next.
"""

from __future__ import annotations

import os

ENABLED = os.environ.get("CUBAM_B200_NVTX", "") not in ("", "0")

#: the range a boundary opens (the stage that follows it)
_NEXT = {"start": "cubam: member scan", "scanned": "cubam: inflate", "inflated": "cubam: record chain",
         "chained": "cubam: record pass"}


def _nvtx():
    import torch

    return torch.cuda.nvtx


def mark(events, name: str, enabled: bool | None = None) -> None:
    """A stage boundary: records ``events``' CUDA event (when given) and, with tracing on, closes the
    open range (not at ``start``) and opens the next stage's (not at ``decoded``)."""
    if events is not None:
        events.mark(name)
    if not (ENABLED if enabled is None else enabled):
        return
    nvtx = _nvtx()
    if name != "start":
        nvtx.range_pop()
    nxt = _NEXT.get(name)
    if nxt is not None:
        nvtx.range_push(nxt)
