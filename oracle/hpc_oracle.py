"""Homopolymer compression of reads, restated in numpy -- TEST
INFRASTRUCTURE ONLY (the checker of the GPU compaction behind opt.hpc).

The reference's GPU_HPCEncoding (gpu_skmgen.cu:145-173) walks each read and
keeps a byte when it differs from the byte before it (the read's first byte is
always kept); bytes are compared as they are, so 'a' and 'A' differ.  The
compressed read then goes through phase 1 like any other.

Pinned to the compiled reference: its CPU phase 1 with HPC on
(cpu_funcs.cpp:253-275) gives this restatement's table of the compressed
reads with each read's last byte dropped, because the reference CPU's
_hpc_encoding returns the last index rather than the length
(cpu_funcs.cpp:92-100); tests/test_hpc.py checks exactly that.  The GPU path,
which this follows, keeps the byte (gpu_skmgen.cu:170).
"""
from __future__ import annotations

import numpy as np


def hpc(reads: np.ndarray, offs: np.ndarray):
    """(reads, offs) CSR -> the homopolymer-compressed CSR."""
    reads = np.asarray(reads, np.uint8)
    offs = np.asarray(offs, np.uint64).astype(np.int64)
    n = len(reads)
    keep = np.ones(n, bool)
    if n > 1:
        keep[1:] = reads[1:] != reads[:-1]
    starts = offs[:-1][offs[:-1] < n]
    keep[starts] = True                     # every read keeps its first byte
    cum = np.concatenate([[0], np.cumsum(keep)])
    return reads[keep].copy(), cum[offs].astype(np.uint64)
