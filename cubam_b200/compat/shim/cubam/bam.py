"""cubam's ``cubam.bam`` names (``src/cubam/bam.py``) from cubam_b200.bam: the record batch, tags,
header, reader, flag constants and the private helpers the applications import (``_strings_at``,
``_string_series``, ``_fnv1a``, ``_record_chain``)."""

from cubam_b200.bam import (
    DUPLICATE,
    MATE_REVERSE,
    MATE_UNMAPPED,
    PAIRED,
    PROPER_PAIR,
    QC_FAIL,
    READ1,
    READ2,
    REVERSE,
    SECONDARY,
    SUPPLEMENTARY,
    UNMAPPED,
    BamHeader,
    RecordBatch,
    Tag,
    _fnv1a,
    _record_chain,
    _string_series,
    _strings_at,
    read_bam,
    unpack_acgt,
)

__all__ = [
    "DUPLICATE", "MATE_REVERSE", "MATE_UNMAPPED", "PAIRED", "PROPER_PAIR", "QC_FAIL", "READ1", "READ2", "REVERSE",
    "SECONDARY", "SUPPLEMENTARY", "UNMAPPED", "BamHeader", "RecordBatch", "Tag", "_fnv1a", "_record_chain",
    "_string_series", "_strings_at", "read_bam", "unpack_acgt",
]
