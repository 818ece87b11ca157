"""cubam's package names over cubam_b200 (``src/cubam/__init__.py:3-7``)."""

from cubam._memory import auto_chunk_bytes, memory_pool
from cubam.bam import BamHeader, RecordBatch, Tag, read_bam
from cubam.bgzf import inflate_chunks

__all__ = ["BamHeader", "RecordBatch", "Tag", "auto_chunk_bytes", "inflate_chunks", "memory_pool", "read_bam"]
