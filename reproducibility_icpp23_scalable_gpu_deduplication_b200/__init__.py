"""B200-native tree-approach incremental-checkpoint deduplicator.

A drop-in for the TreeDeduplicator of TauferLab/Reproducibility_ICPP23_Scalable_GPU_Deduplication:
hand-written sm_100a CUDA kernels behind the C ABI in include/b200dedup.h
(libb200dedup.so, built in this directory), with this Python mirror of its interface.
"""
from ._lib import HASH_MD5, HASH_MURMUR3, B2DError, lib, lib_path  # noqa: F401
from .tree import ListDeduplicator, TreeDeduplicator, hash_chunks, parse_header  # noqa: F401
from .batch import CheckpointBatch  # noqa: F401

__all__ = ["TreeDeduplicator", "ListDeduplicator", "CheckpointBatch", "hash_chunks", "parse_header", "HASH_MURMUR3", "HASH_MD5", "B2DError", "lib",
           "lib_path"]
