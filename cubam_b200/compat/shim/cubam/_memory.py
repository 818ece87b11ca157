"""cubam's ``cubam._memory`` names (``src/cubam/_memory.py:11-45``) from cubam_b200."""

from cubam_b200._memory import _CHUNK_SHARE, auto_chunk_bytes, memory_pool

__all__ = ["_CHUNK_SHARE", "auto_chunk_bytes", "memory_pool"]
