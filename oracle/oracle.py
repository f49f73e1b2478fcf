"""ctypes bindings for the test oracles -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker or as the timed CPU baseline.  The
product package (rapidgkc_b200) never imports it and has no CPU fallback.

Two oracles are exposed:

* ``Oracle`` -- the C restatement in oracle/gkc_oracle.c of the reference
  algorithm (each C function cites the reference file:line it follows);
* ``RefOracle`` -- the reference's own CPU path (cpu_funcs.cpp compiled from
  the reference tree by oracle/Makefile into oracle/_ref/libgkc_ref.so, and
  with -DLONGERKMER into oracle/_ref/libgkc_ref_long.so for k > 32).

For k <= 32 k-mers are u64 arrays; for 32 < k <= 64 they are (n, 2) u64
arrays of (low word, high word), the layout of the reference's 128-bit
T_kmer (types.h:34-35), ordered as 128-bit values.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def _ptr_or_null(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """The C restatement (oracle/liboracle.so)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = C.CDLL(path)
        L.orc_filter_default.argtypes = [C.c_uint32, C.c_int]
        L.orc_filter_default.restype = C.c_int
        L.orc_kmer_keys.argtypes = [_u8p, C.c_int64, C.c_int, C.c_int, C.c_void_p, _u32p]
        L.orc_kmer_keys.restype = C.c_int64
        L.orc_skm_split.argtypes = [_u8p, C.c_int64, C.c_int, C.c_int, C.c_void_p, _i64p, _u32p]
        L.orc_skm_split.restype = C.c_int64
        L.orc_skmgen.argtypes = [_u8p, _u64p, C.c_int64, C.c_int, C.c_int, C.c_uint32, C.c_void_p,
                                 _u64p, _u64p, _u64p, C.c_void_p, C.c_void_p]
        L.orc_skmgen.restype = C.c_int64
        L.orc_extract.argtypes = [_u8p, C.c_uint64, C.c_int, C.c_void_p]
        L.orc_extract.restype = C.c_int64
        L.orc_count.argtypes = [_u64p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_int64)]
        L.orc_count.restype = C.c_int64
        L.orc_revcomp.argtypes = [C.c_uint64, C.c_int]
        L.orc_revcomp.restype = C.c_uint64
        L.orc_sort_u64.argtypes = [_u64p, C.c_int64]
        L.orc_sort_u64.restype = None
        L.orc_extract_wide.argtypes = [_u8p, C.c_uint64, C.c_int, C.c_void_p]
        L.orc_extract_wide.restype = C.c_int64
        L.orc_count_wide.argtypes = [_u64p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                     C.POINTER(C.c_int64)]
        L.orc_count_wide.restype = C.c_int64

    # -- phase 1 ---------------------------------------------------------
    def kmer_keys(self, read: bytes, k: int, p: int, lut=None) -> np.ndarray:
        a = np.frombuffer(read, np.uint8).copy()
        out = np.zeros(max(0, len(a) - k + 1), np.uint32)
        if len(a) >= k:
            self.lib.orc_kmer_keys(a, len(a), k, p, _ptr_or_null(lut), out)
        return out

    def skm_split(self, read: bytes, k: int, p: int, lut=None):
        a = np.frombuffer(read, np.uint8).copy()
        offs = np.zeros(len(a) + 2, np.int64)
        mm = np.zeros(len(a) + 1, np.uint32)
        n = self.lib.orc_skm_split(a, len(a), k, p, _ptr_or_null(lut), offs, mm)
        return offs[: n + 1].copy(), mm[:n].copy()

    def skmgen(self, reads: np.ndarray, offs: np.ndarray, k: int, p: int, P: int, lut=None):
        """Returns (part_bytes, part_skms, part_kmers, part_offsets, stream):
        each partition's superkmers in read order, concatenated by partition."""
        reads = np.ascontiguousarray(reads, np.uint8)
        offs = np.ascontiguousarray(offs, np.uint64)
        n = len(offs) - 1
        pb = np.zeros(P, np.uint64); ps = np.zeros(P, np.uint64); pk = np.zeros(P, np.uint64)
        self.lib.orc_skmgen(reads, offs, n, k, p, P, _ptr_or_null(lut), pb, ps, pk, None, None)
        po = np.zeros(P + 1, np.uint64)
        po[1:] = np.cumsum(pb)
        out = np.zeros(int(po[-1]), np.uint8)
        cur = po[:-1].copy()
        self.lib.orc_skmgen(reads, offs, n, k, p, P, _ptr_or_null(lut), pb, ps, pk,
                            out.ctypes.data_as(C.c_void_p), cur.ctypes.data_as(C.c_void_p))
        return pb, ps, pk, po, out

    # -- phase 2 ---------------------------------------------------------
    def extract(self, stream: np.ndarray, k: int) -> np.ndarray:
        stream = np.ascontiguousarray(stream, np.uint8)
        fn = self.lib.orc_extract_wide if k > 32 else self.lib.orc_extract
        n = fn(stream, len(stream), k, None)
        if n < 0:
            raise ValueError("malformed superkmer stream")
        out = np.zeros((n, 2) if k > 32 else n, np.uint64)
        fn(stream, len(stream), k, out.ctypes.data_as(C.c_void_p))
        return out

    def count(self, keys: np.ndarray, cmin: int = 1, cmax: int = 0xFFFFFFFF):
        """Sort + RLE + threshold.  Returns (kmers, counts, n_distinct); keys
        of shape (n, 2) are 128-bit (low, high) pairs."""
        keys = np.array(keys, np.uint64, copy=True)
        wide = keys.ndim == 2
        n = len(keys)
        ok = np.zeros(keys.shape, np.uint64)
        oc = np.zeros(n, np.uint32)
        d = C.c_int64(0)
        fn = self.lib.orc_count_wide if wide else self.lib.orc_count
        w = fn(keys.reshape(-1) if wide else keys, n, cmin, cmax, ok.ctypes.data_as(C.c_void_p),
               oc.ctypes.data_as(C.c_void_p), C.byref(d))
        return ok[:w].copy(), oc[:w].copy(), int(d.value)

    def count_reads(self, reads, offs, k, p, P, cmin=1, cmax=0xFFFFFFFF, lut=None):
        """Whole path: returns (kmers, counts, n_distinct, part_kmers) with the
        output ordered by partition, ascending key within a partition."""
        pb, ps, pk, po, stream = self.skmgen(reads, offs, k, p, P, lut)
        ks, cs, dist = [], [], 0
        for i in range(P):
            keys = self.extract(stream[int(po[i]):int(po[i + 1])], k)
            a, b, d = self.count(keys, cmin, cmax)
            ks.append(a); cs.append(b); dist += d
        return np.concatenate(ks), np.concatenate(cs), dist, pk

    def revcomp(self, x: int, k: int) -> int:
        return int(self.lib.orc_revcomp(x, k))


class RefOracle:
    """The reference's own CPU path (oracle/_ref/libgkc_ref.so; with
    ``wide=True`` its 128-bit LONGERKMER build, oracle/_ref/libgkc_ref_long.so,
    for k <= 64)."""

    def __init__(self, path: str | None = None, wide: bool = False):
        path = path or os.path.join(HERE, "_ref", "libgkc_ref_long.so" if wide else "libgkc_ref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        L = self.lib = C.CDLL(path)
        L.ref_kmer_bits.argtypes = []
        L.ref_kmer_bits.restype = C.c_int
        self.wide = L.ref_kmer_bits() == 128
        L.ref_gen_skm_offs.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _i32p, _u32p]
        L.ref_gen_skm_offs.restype = C.c_int
        L.ref_phase1.argtypes = [_u8p, _u64p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int,
                                 _u64p, _u64p, _u64p]
        L.ref_phase1.restype = C.c_void_p
        L.ref_phase1_hpc.argtypes = [_u8p, _u64p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     _u64p, _u64p, _u64p]
        L.ref_phase1_hpc.restype = C.c_void_p
        L.ref_part_bytes.argtypes = [C.c_void_p, C.c_int, _u8p]
        L.ref_part_bytes.restype = C.c_int64
        L.ref_count_bytes.argtypes = [_u8p, C.c_uint64, C.c_uint64, C.c_int, C.c_uint32, C.c_uint32,
                                      C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
        L.ref_count_bytes.restype = C.c_int64
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_free.restype = None
        L.ref_run.argtypes = [_u8p, _u64p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int,
                              C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ref_run.restype = C.c_int64
        L.ref_digest.argtypes = [_u8p, _u64p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint32,
                                 C.c_uint32, _u64p]
        L.ref_digest.restype = C.c_int

    def gen_skm_offs(self, read: bytes, k: int, p: int):
        offs = np.zeros(len(read) + 2, np.int32)
        mm = np.zeros(len(read) + 1, np.uint32)
        n = self.lib.ref_gen_skm_offs(read, len(read), k, p, offs, mm)
        return offs[: n + 1].copy(), mm[:n].copy()

    def phase1(self, reads, offs, k, p, P, threads=1, hpc=False):
        """Returns (part_bytes, part_skms, part_kmers, list of per-partition byte arrays).
        hpc: the reference's CPU homopolymer compression (every read must stay
        at least k + 1 bytes long after it)."""
        reads = np.ascontiguousarray(reads, np.uint8)
        offs = np.ascontiguousarray(offs, np.uint64)
        pb = np.zeros(P, np.uint64); ps = np.zeros(P, np.uint64); pk = np.zeros(P, np.uint64)
        h = self.lib.ref_phase1_hpc(reads, offs, len(offs) - 1, k, p, P, threads, int(hpc), pb, ps, pk)
        try:
            parts = []
            for i in range(P):
                buf = np.zeros(int(pb[i]) + 1, np.uint8)
                n = self.lib.ref_part_bytes(h, i, buf)
                parts.append(buf[:n].copy())
        finally:
            self.lib.ref_free(h)
        return pb, ps, pk, parts

    def count_bytes(self, stream, n_kmers, k, cmin=1, cmax=0xFFFFFFFF):
        stream = np.ascontiguousarray(stream, np.uint8)
        if (k > 32) != self.wide:
            raise ValueError(f"k={k} needs the {'128' if k > 32 else '64'}-bit reference build")
        ok = np.zeros((max(1, n_kmers), 2) if self.wide else max(1, n_kmers), np.uint64)
        oc = np.zeros(max(1, n_kmers), np.uint32)
        d = C.c_int64(0)
        w = self.lib.ref_count_bytes(stream if len(stream) else np.zeros(1, np.uint8), len(stream),
                                     n_kmers, k, cmin, cmax, ok.ctypes.data_as(C.c_void_p),
                                     oc.ctypes.data_as(C.c_void_p), C.byref(d))
        if w < 0:
            raise ValueError("reference extraction disagreed with the partition k-mer count")
        return ok[:w].copy(), oc[:w].copy(), int(d.value)

    def count_reads(self, reads, offs, k, p, P, cmin=1, cmax=0xFFFFFFFF, threads=1, hpc=False):
        """Whole reference path; output ordered by partition, ascending within."""
        pb, ps, pk, parts = self.phase1(reads, offs, k, p, P, threads, hpc)
        ks, cs, dist = [], [], 0
        for i in range(P):
            a, b, d = self.count_bytes(parts[i], int(pk[i]), k, cmin, cmax)
            ks.append(a); cs.append(b); dist += d
        return np.concatenate(ks), np.concatenate(cs), dist, pk

    def digest(self, reads, offs, k, p, P, threads=1, cmin=1, cmax=0xFFFFFFFF) -> dict:
        """Order-independent digest of the reference's thresholded table
        (ref_digest): kept, distinct, xor, sum_kc, sum_c, instances.  A
        128-bit k-mer enters as low ^ high * 0x9E3779B97F4A7C15."""
        reads = np.ascontiguousarray(reads, np.uint8)
        offs = np.ascontiguousarray(offs, np.uint64)
        out = np.zeros(6, np.uint64)
        if self.lib.ref_digest(reads, offs, len(offs) - 1, k, p, P, threads, cmin, cmax, out) != 0:
            raise ValueError("reference extraction disagreed with the partition k-mer count")
        return dict(zip(("kept", "distinct", "xor", "sum_kc", "sum_c", "instances"), (int(x) for x in out)))

    def run(self, reads, offs, k, p, P, threads):
        """Timed CPU-only reference pipeline.  Returns (distinct, t_phase1, t_phase2)."""
        reads = np.ascontiguousarray(reads, np.uint8)
        offs = np.ascontiguousarray(offs, np.uint64)
        t1 = C.c_double(0); t2 = C.c_double(0)
        d = self.lib.ref_run(reads, offs, len(offs) - 1, k, p, P, threads, C.byref(t1), C.byref(t2))
        return int(d), t1.value, t2.value


def ref_load_reads(path: str, buffer_mb: int = 1, timeout: float = 120.0) -> list:
    """The reads of a FASTQ / FASTA file (FASTA when the name ends in 'a') as
    the reference's ReadLoader extracts them (fileloader.hpp:51-545), run as
    the program oracle/_ref/ref_load_reads in a process of its own."""
    import subprocess
    import tempfile
    exe = os.path.join(HERE, "_ref", "ref_load_reads")
    if not os.path.exists(exe):
        raise FileNotFoundError(f"{exe} missing: run `make -C oracle ref` where the reference tree exists")
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "reads.bin")
        p = subprocess.run([exe, path, str(buffer_mb), out], capture_output=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference loader failed ({p.returncode}): {p.stderr[-500:]!r}")
        b = open(out, "rb").read()
    n = int(np.frombuffer(b[:8], np.uint64)[0])
    offs = np.frombuffer(b[8:8 + 8 * (n + 1)], np.uint64).astype(np.int64)
    data = b[8 + 8 * (n + 1):]
    return [data[offs[i]:offs[i + 1]] for i in range(n)]
