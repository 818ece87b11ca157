"""BAI index and region queries on the CPU: TEST INFRASTRUCTURE ONLY.

cubam has no BAI support (docs/reading.md:52-53, docs/development.md:52), so there is no
reference code to follow; this restates the index of the SAM/BAM specification (SAMv1, section
5.2 "The BAI index format for BAM files", section 5.3 "C source code for computing bin number
and overlapping bins") with plain Python loops, for small inputs:

- bin of a record = reg2bin(beg, end) over [pos, end) (end = the alignment end, at least
  pos + 1), 6 levels of 2^29 / 2^26 / ... / 2^14 bases;
- chunks of a bin = runs of consecutive records (file order) with the same bin, as
  [virtual offset of the first record, virtual offset just past the last);
- linear index = per 16 kb window the smallest virtual offset of a record overlapping it,
  empty windows taking the value of the window before, and empty windows before the first
  record's window the reference's first record offset (the pseudo-bin's start), as htslib
  fills them;
- pseudo-bin 37450 per reference: [first record's offset, end of the last], (mapped, unmapped);
- records without a reference (ref < 0) are counted in n_no_coor.

Two chunks of a bin are then merged when the first ends in the BGZF block where the second starts
(the end's block offset at or past the start's), as htslib does to keep the index small.
"""

from __future__ import annotations

import struct

import numpy as np

PSEUDO_BIN = 37450


def reg2bin(beg: int, end: int) -> int:
    """The bin of [beg, end) (SAMv1 5.3)."""
    end -= 1
    if beg >> 14 == end >> 14:
        return ((1 << 15) - 1) // 7 + (beg >> 14)
    if beg >> 17 == end >> 17:
        return ((1 << 12) - 1) // 7 + (beg >> 17)
    if beg >> 20 == end >> 20:
        return ((1 << 9) - 1) // 7 + (beg >> 20)
    if beg >> 23 == end >> 23:
        return ((1 << 6) - 1) // 7 + (beg >> 23)
    if beg >> 26 == end >> 26:
        return ((1 << 3) - 1) // 7 + (beg >> 26)
    return 0


def reg2bins(beg: int, end: int) -> list[int]:
    """The bins that may hold records overlapping [beg, end) (SAMv1 5.3)."""
    end -= 1
    out = [0]
    for first, shift in ((1, 26), (9, 23), (73, 20), (585, 17), (4681, 14)):
        out.extend(range(first + (beg >> shift), first + (end >> shift) + 1))
    return out


def record_end(pos: int, end: int) -> int:
    """The end used by the index: the alignment end, at least one base past pos."""
    return max(int(end), int(pos) + 1)


def build(n_ref: int, ref, pos, end, flag, voff, voff_next) -> bytes:
    """BAI bytes of records in file order: voff[i] starts record i, voff_next[i] is just past it."""
    refs = [dict(bins={}, lin={}, beg=None, last=None, mapped=0, unmapped=0) for _ in range(n_ref)]
    n_no_coor = 0
    cur = None  # (ref, bin) of the open chunk and its chunk list entry
    for i in range(len(ref)):
        r, p = int(ref[i]), int(pos[i])
        if r < 0:
            n_no_coor += 1
            cur = None
            continue
        e = record_end(p, end[i])
        b = reg2bin(p, e)
        R = refs[r]
        if cur is not None and cur[0] == (r, b):
            cur[1][1] = int(voff_next[i])
        else:
            chunk = [int(voff[i]), int(voff_next[i])]
            R["bins"].setdefault(b, []).append(chunk)
            cur = ((r, b), chunk)
        for w in range(p >> 14, ((e - 1) >> 14) + 1):
            if w not in R["lin"]:
                R["lin"][w] = int(voff[i])
        if R["beg"] is None:
            R["beg"] = int(voff[i])
        R["last"] = int(voff_next[i])
        if int(flag[i]) & 4:
            R["unmapped"] += 1
        else:
            R["mapped"] += 1
    for R in refs:
        for b, chunks in R["bins"].items():
            merged = [chunks[0]]
            for c in chunks[1:]:
                if merged[-1][1] >> 16 >= c[0] >> 16:
                    merged[-1] = [merged[-1][0], max(merged[-1][1], c[1])]
                else:
                    merged.append(c)
            R["bins"][b] = merged
    out = [b"BAI\x01", struct.pack("<i", n_ref)]
    for R in refs:
        bins = sorted(R["bins"].items())
        n_bin = len(bins) + (1 if R["beg"] is not None else 0)
        out.append(struct.pack("<i", n_bin))
        for b, chunks in bins:
            out.append(struct.pack("<Ii", b, len(chunks)))
            for c in chunks:
                out.append(struct.pack("<QQ", c[0], c[1]))
        if R["beg"] is not None:
            out.append(struct.pack("<Ii", PSEUDO_BIN, 2))
            out.append(struct.pack("<QQQQ", R["beg"], R["last"], R["mapped"], R["unmapped"]))
        if R["lin"]:
            n_intv = max(R["lin"]) + 1
            lin, prev = [], R["beg"] if R["beg"] is not None else 0
            for w in range(n_intv):
                prev = R["lin"].get(w, prev)
                lin.append(prev)
            out.append(struct.pack("<i", n_intv))
            out.append(struct.pack(f"<{n_intv}Q", *lin))
        else:
            out.append(struct.pack("<i", 0))
    out.append(struct.pack("<Q", n_no_coor))
    return b"".join(out)


def overlaps(ref, pos, end, r: int, beg: int, stop: int) -> np.ndarray:
    """Records of reference r overlapping [beg, stop)."""
    ref, pos, end = (np.asarray(x, np.int64) for x in (ref, pos, end))
    e = np.maximum(end, pos + 1)
    return (ref == r) & (pos < stop) & (e > beg)
