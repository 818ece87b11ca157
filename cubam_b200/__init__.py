"""Read BAM files on the B200, as columns: cubam's reader API on hand-written sm_100a kernels."""

from cubam_b200._memory import auto_chunk_bytes, memory_pool
from cubam_b200.bam import BamHeader, RecordBatch, Tag, read_bam, unpack_acgt
from cubam_b200.bgzf import inflate_chunks
from cubam_b200.strings import StringColumn

__all__ = [
    "BamHeader",
    "RecordBatch",
    "StringColumn",
    "Tag",
    "auto_chunk_bytes",
    "inflate_chunks",
    "memory_pool",
    "read_bam",
    "unpack_acgt",
]
