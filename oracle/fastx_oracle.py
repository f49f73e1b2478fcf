"""FASTQ / FASTA record rules, restated in plain Python -- TEST
INFRASTRUCTURE ONLY (the checker of the GPU record scanner; small inputs).

FASTQ follows the reference loader (fileloader.hpp:201-232): the text is cut
at '\\n'; line i of the text has phase (state + i) mod 4, and the lines of
phase 1 are the reads (fileloader.hpp:222 `is_read_line == 1`, with
`flag_mask = 0b11`, :203).  The phase after the text is returned, as the
loader carries `is_read_line` from one buffer to the next.  A read line is
kept whole except for '\\r' bytes (the reference keeps a trailing '\\r' in the
read, where it becomes an invalid base; dropping it keeps CRLF files exact).

Pinned to the compiled reference: tests/test_fastx.py runs the reference's
own ReadLoader (as oracle/_ref/ref_load_reads) on multi-megabyte FASTQ and
single-line FASTA files read in 1 MB buffers, and its reads equal these, in
order (empty reads aside, which the loader skips and which hold no k-mer).

FASTA: a record is a '>' header line and the sequence lines up to the next
header, concatenated without '\\r'.  The reference loader instead takes every
second line (`flag_mask = 0b1`, :203), which is right only for single-line
FASTA; on such text both rules give the same reads.  Text that starts with
sequence lines yields those bases as a first read (a record continued from
earlier text).
"""
from __future__ import annotations

import numpy as np


def parse_fastx(text: bytes, fmt: str = "fastq", state: int = 0):
    """Returns (reads as a list of bytes, state after the text).  Reads that
    start at a phase-0 newline at the very end of the text are empty."""
    if not text:
        return [], (state if fmt == "fastq" else 0)
    lines = text.split(b"\n")
    reads = []
    if fmt == "fastq":
        for i, line in enumerate(lines):
            if (state + i) & 3 == 1:
                reads.append(line.replace(b"\r", b""))
        return reads, (state + len(lines) - 1) & 3
    cur = None
    for i, line in enumerate(lines):
        if line.startswith(b">"):
            if cur is not None:
                reads.append(cur)
            cur = b""
        else:
            if cur is None:          # text that starts inside a record
                cur = b""
            cur += line.replace(b"\r", b"")
    if cur is not None:
        reads.append(cur)
    return reads, 0


def csr(reads):
    """(uint8 bases, uint64 offsets) of a list of reads."""
    offs = np.zeros(len(reads) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in reads]) if reads else []
    return np.frombuffer(b"".join(reads), np.uint8).copy(), offs
