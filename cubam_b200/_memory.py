"""GPU memory: how much to read at a time, and the pool.

Mirrors ``src/cubam/_memory.py``: the chunk policy is the same rule (halved
while 64 chunks do not fit in free GPU memory, never below 32 MB) from a
ceiling of 1 GB instead of 256 MB: a B200's 180 GB hold 64 chunks of 1 GB, and
a chunk of 1 GB holds about 39,000 BGZF members, enough for the two-kernel
inflater (one member per lane) to run, while chunks stay small enough for the
host reads of the next ones to overlap the GPU work (page cache to pinned
memory ran at 29 GB/s with 1 GB chunks and 25 GB/s with 2 GB chunks, 16
threads).  Below 32 GB of free memory the sizes are cubam's (64 MB on 8 GB,
128 MB on 16 GB, 256 MB on 24 GB).
Buffers come from PyTorch's caching allocator, which is already a
stream-ordered pool, so :func:`memory_pool` only has to exist for callers
written against cubam.
"""

from __future__ import annotations

from contextlib import contextmanager

import torch

#: Peak GPU memory of the reader is a small multiple of the compressed chunk
_CHUNK_SHARE = 64


def auto_chunk_bytes() -> int:
    """Compressed bytes to read per chunk (``src/cubam/_memory.py:11-23``)."""
    free, _ = torch.cuda.mem_get_info()
    size = 1 << 30
    while size > 32 << 20 and size * _CHUNK_SHARE > free:
        size //= 2
    return size


@contextmanager
def memory_pool():
    """Kept for cubam's API (``src/cubam/_memory.py:27-45``): PyTorch's caching allocator is the pool."""
    yield
