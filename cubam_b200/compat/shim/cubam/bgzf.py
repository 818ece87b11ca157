"""cubam's ``cubam.bgzf`` names (``src/cubam/bgzf.py``) from cubam_b200: the chunked reader and
inflater (``inflate_chunks``, ``_inflate``, ``_inflate_blocks``, ``_ChunkReader``) and the write
side (``BgzfWriter``, ``_bgzf_compress``, ``_deflate_spans``, the checksums, ``BLOCK_DATA``,
``EOF_BLOCK``)."""

from cubam_b200.bgzf import (
    BLOCK_DATA,
    EOF_BLOCK,
    BgzfWriter,
    _adler32_spans,
    _bgzf_compress,
    _ChunkReader,
    _crc32_spans,
    _deflate_spans,
    _inflate,
    _inflate_blocks,
    inflate_chunks,
)

#: Largest ISIZE of a BGZF member (``src/cubam/bgzf.py:35``)
_MAX_ISIZE = 1 << 16

__all__ = [
    "BLOCK_DATA", "EOF_BLOCK", "BgzfWriter", "_MAX_ISIZE", "_adler32_spans", "_bgzf_compress", "_ChunkReader",
    "_crc32_spans", "_deflate_spans", "_inflate", "_inflate_blocks", "inflate_chunks",
]
