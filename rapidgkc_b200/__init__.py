"""B200-native k-mer counter with RapidGKC's interface.

Reads -> 2-bit packing -> canonical minimizers -> superkmers in per-partition
device buffers -> canonical uint64 k-mers -> count (LSD radix sort + run-length
reduction, or an L2-resident open-addressing hash) -> [min, max] threshold, all
in hand-written sm_100a CUDA behind the C ABI of include/gkc_capi.h.
"""
from .capi import KmerCounter, GkcError, load_library, UINT32_MAX  # noqa: F401

__all__ = ["KmerCounter", "GkcError", "load_library", "UINT32_MAX"]
