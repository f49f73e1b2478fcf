"""Seeded synthetic workloads (libgkc_synth.so) with the shapes the counter is
specified on.  No public dataset is available here, so these stand in for real
sequencing data: genome size, GC content, repeat families, low-complexity runs,
read length distribution, strand and substitution rate follow each workload's
description, and every draw is reproducible from the seed.

Workloads (``make_workload(name, scale)``; ``scale`` shrinks genome and read
count together, coverage unchanged):

* ``uniform_5m``    5 Mbp i.i.d. uniform genome, 1M x 150 bp reads (30x), 0.5% errors
* ``bacterial_100m`` 100 Mbp, GC 41%, 10% repeats (200 families of 1-5 kb at 2%
  divergence), 20M x 150 bp reads (30x, 3 Gbp), 0.3% errors
* ``mixed_100m``    the 100 Mbp genome; 80% of bases from 150 bp reads (0.3%),
  20% from log-normal long reads (median 8 kb, clipped 1-50 kb, 5% errors)
* ``skewed_200m``   200 Mbp, GC 38%, 8% low-complexity runs of 50-2000 bp
  (poly-A, (AT)n, (CAG)n), 15% repeats, 40M x 150 bp reads (30x), 0.3% errors
* ``human_3g``      3.1 Gbp, GC 41%, 50% repeats (1-20% divergence), 150 bp
  reads at 30x (streamed in batches by the caller)
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libgkc_synth.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: run `python -m rapidgkc_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, u64, i64, i32, d = C.c_void_p, C.c_uint64, C.c_int64, C.c_int, C.c_double
        L.gkc_synth_genome.argtypes = [u64, i64, d, d, i32, i32, i32, d, d, d, i32, i32, vp, i32]
        L.gkc_synth_reads.argtypes = [vp, i64, u64, i64, i32, d, i32, vp, vp, i32]
        L.gkc_synth_long_read_lengths.argtypes = [u64, i64, d, d, i64, i64, vp]
        L.gkc_synth_reads_var.argtypes = [vp, i64, u64, u64, i64, vp, d, i32, vp, i32]
        for f in ("gkc_synth_genome", "gkc_synth_reads", "gkc_synth_long_read_lengths", "gkc_synth_reads_var"):
            getattr(L, f).restype = i32
        _lib = L
    return _lib


@dataclass
class GenomeSpec:
    length: int
    gc: float = 0.5
    repeat_frac: float = 0.0
    n_families: int = 0
    fam_min: int = 1000
    fam_max: int = 5000
    div_min: float = 0.02
    div_max: float = 0.02
    lowcomp_frac: float = 0.0
    lc_min: int = 50
    lc_max: int = 2000


def genome(spec: GenomeSpec, seed: int, threads: int = 0) -> np.ndarray:
    g = np.empty(spec.length, np.uint8)
    rc = _load().gkc_synth_genome(seed, spec.length, spec.gc, spec.repeat_frac, spec.n_families, spec.fam_min,
                                  spec.fam_max, spec.div_min, spec.div_max, spec.lowcomp_frac, spec.lc_min,
                                  spec.lc_max, g.ctypes.data_as(C.c_void_p), threads)
    if rc:
        raise ValueError(f"gkc_synth_genome failed ({rc})")
    return g


def _alloc(n, dtype, pinned):
    if pinned:
        import torch
        return torch.empty(int(n), dtype={np.uint8: torch.uint8, np.uint64: torch.int64}[dtype],
                           pin_memory=True).numpy().view(dtype)
    return np.empty(int(n), dtype)


def short_reads(g: np.ndarray, n_reads: int, read_len: int, err: float, seed: int, both_strands=True,
                pinned=False, threads: int = 0):
    reads = _alloc(n_reads * read_len, np.uint8, pinned)
    offs = _alloc(n_reads + 1, np.uint64, pinned)
    rc = _load().gkc_synth_reads(g.ctypes.data_as(C.c_void_p), len(g), seed, n_reads, read_len, err,
                                 int(both_strands), reads.ctypes.data_as(C.c_void_p),
                                 offs.ctypes.data_as(C.c_void_p), threads)
    if rc:
        raise ValueError(f"gkc_synth_reads failed ({rc})")
    return reads, offs


def long_read_lengths(n: int, median: float, sigma: float, lmin: int, lmax: int, seed: int) -> np.ndarray:
    out = np.empty(n, np.int64)
    rc = _load().gkc_synth_long_read_lengths(seed, n, median, sigma, lmin, lmax, out.ctypes.data_as(C.c_void_p))
    if rc:
        raise ValueError("gkc_synth_long_read_lengths failed")
    return out


def reads_with_lengths(g: np.ndarray, lens: np.ndarray, err: float, seed: int, stream: int = 1,
                       both_strands=True, pinned=False, threads: int = 0):
    offs = _alloc(len(lens) + 1, np.uint64, pinned)
    offs[0] = 0
    np.cumsum(lens, out=offs[1:])
    reads = _alloc(int(offs[-1]), np.uint8, pinned)
    rc = _load().gkc_synth_reads_var(g.ctypes.data_as(C.c_void_p), len(g), seed, stream, len(lens),
                                     offs.ctypes.data_as(C.c_void_p), err, int(both_strands),
                                     reads.ctypes.data_as(C.c_void_p), threads)
    if rc:
        raise ValueError(f"gkc_synth_reads_var failed ({rc})")
    return reads, offs


def concat(parts, pinned=False):
    total = sum(len(r) for r, _ in parts)
    nr = sum(len(o) - 1 for _, o in parts)
    reads = _alloc(total, np.uint8, pinned)
    offs = _alloc(nr + 1, np.uint64, pinned)
    ro = 0
    oo = 0
    offs[0] = 0
    for r, o in parts:
        reads[ro:ro + len(r)] = r
        offs[oo + 1:oo + len(o)] = o[1:] + ro
        ro += len(r)
        oo += len(o) - 1
    return reads, offs


WORKLOADS = {
    "uniform_5m": dict(genome=GenomeSpec(5_000_000, gc=0.5), n_reads=1_000_000, err=0.005, seed=101),
    "bacterial_100m": dict(genome=GenomeSpec(100_000_000, gc=0.41, repeat_frac=0.10, n_families=200),
                           n_reads=20_000_000, err=0.003, seed=202),
    "mixed_100m": dict(genome=GenomeSpec(100_000_000, gc=0.41, repeat_frac=0.10, n_families=200),
                       n_reads=16_000_000, err=0.003, long_frac=0.2, long_err=0.05, seed=202),
    "skewed_200m": dict(genome=GenomeSpec(200_000_000, gc=0.38, repeat_frac=0.15, n_families=500,
                                          div_min=0.02, div_max=0.10, lowcomp_frac=0.08),
                        n_reads=40_000_000, err=0.003, seed=404),
    "human_3g": dict(genome=GenomeSpec(3_100_000_000, gc=0.41, repeat_frac=0.50, n_families=5000, fam_min=300,
                                       fam_max=6000, div_min=0.01, div_max=0.20),
                     n_reads=620_000_000, err=0.003, seed=505),
}


def make_workload(name: str, scale: float = 1.0, pinned: bool = False, seed: int | None = None,
                  threads: int = 0, read_len: int = 150, read_fraction: float = 1.0, read_seed: int = 0):
    """Returns (reads uint8, offs uint64) for a named workload at `scale`.
    `read_fraction` keeps the genome and samples only that fraction of the
    reads (a bounded sample of the same workload); `read_seed` draws another
    read set from the same genome."""
    w = WORKLOADS[name]
    spec = GenomeSpec(**{**w["genome"].__dict__})
    spec.length = max(10_000, int(spec.length * scale))
    s = w["seed"] if seed is None else seed
    g = genome(spec, s, threads)
    s += 7919 * read_seed
    n = max(1, int(w["n_reads"] * scale * read_fraction))
    if "long_frac" not in w:
        return short_reads(g, n, read_len, w["err"], s + 1, pinned=pinned, threads=threads)
    short = short_reads(g, n, read_len, w["err"], s + 1, threads=threads)
    long_bases = int(len(short[0]) * w["long_frac"] / (1 - w["long_frac"]))
    lmax = min(50_000, len(g))
    lens = long_read_lengths(max(1, long_bases // 9000 + 1), 8000.0, 0.5, min(1000, lmax), lmax, s + 2)
    lens = lens[np.cumsum(lens) <= max(long_bases, int(lens[0]))]
    long = reads_with_lengths(g, lens, w["long_err"], s + 3, threads=threads)
    return concat([short, long], pinned=pinned)
