"""Regenerates the golden fixtures in this directory from the reference itself.

Run where the reference source tree exists (the reference's own CPU path is
compiled from it by oracle/Makefile into oracle/_ref/libgkc_ref.so, and its
128-bit LONGERKMER build, used for k > 32, into oracle/_ref/libgkc_ref_long.so):

    make -C oracle && python tests/golden/make_golden.py [case ...]

(no case names: every fixture).

Fixtures (inputs and the reference's outputs, all seeded):
  skm_test_vector.json  the reference's own known answer (cpu_funcs.cpp:654-676):
                        superkmer offsets and minimizers of one read, k=10, p=5
  <case>.npz            reads (CSR), k, p, P, the reference's per-partition
                        bytes/superkmers/k-mers (SKMStoreNoncon counters), a
                        SHA-256 of each partition's sorted superkmer multiset,
                        and the full sorted (k-mer, count) table (cmin = 1);
                        for k > 32 the k-mers are (n, 2) u64 (low, high) pairs
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import RefOracle  # noqa: E402


def split_superkmers(stream: np.ndarray) -> list[bytes]:
    """Splits a partition stream into superkmers: a first byte, full bytes,
    and a terminal non-full byte (the layout of cpu_funcs.cpp:238-244)."""
    out, i, n = [], 0, len(stream)
    while i < n:
        j = i + 1
        while j < n and (stream[j] >> 6) == 3:
            j += 1
        out.append(bytes(stream[i:j + 1]))
        i = j + 1
    return out


def partition_digest(stream: np.ndarray) -> str:
    h = hashlib.sha256()
    for s in sorted(split_superkmers(stream)):
        h.update(len(s).to_bytes(4, "little"))
        h.update(s)
    return h.hexdigest()


def rng_reads(seed, genome_len, n_reads, read_len, err, alphabet=b"ACGT"):
    r = np.random.default_rng(seed)
    g = np.frombuffer(alphabet, np.uint8)[r.integers(0, len(alphabet), genome_len)]
    comp = np.zeros(256, np.uint8)
    for a, b in zip(b"ACGTN", b"TGCAN"):
        comp[a] = b
    reads, offs = [], [0]
    for _ in range(n_reads):
        L = read_len if np.isscalar(read_len) else int(r.integers(read_len[0], read_len[1] + 1))
        L = min(L, genome_len)
        pos = int(r.integers(0, genome_len - L + 1))
        s = g[pos:pos + L].copy()
        if r.integers(0, 2):
            s = comp[s[::-1]]
        m = r.random(L) < err
        s[m] = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, int(m.sum()))]
        reads.append(s)
        offs.append(offs[-1] + L)
    return np.concatenate(reads).astype(np.uint8), np.array(offs, np.uint64)


def edge_reads(seed):
    """Reads exercising the reference's edge cases: shorter than k, exactly k,
    empty, N and U bases, lower case, poly-A runs and a long read."""
    r = np.random.default_rng(seed)
    parts = []
    for L in [0, 1, 10, 24, 25, 26, 27, 30, 31, 32, 33, 150, 151, 152, 997]:
        parts.append(bytes(np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, L)]))
    parts.append(b"A" * 300)
    parts.append(b"AT" * 200)
    parts.append(b"CAG" * 120)
    parts.append(b"ACGTNACGTN" * 20)
    parts.append(b"acgtgtcagctagctagcatcgatcgactacgactagcatcgactacgatcg" * 3)
    parts.append(b"ACGUACGUUUGACGUAGCUAGCAUGCAUCGUACGAUCGUAGCUAGCUAGCAUCGAUCGA")
    parts.append(bytes(np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, 5000)]))
    parts.append(b"G" * 40 + b"T" * 40 + b"C" * 40)
    reads = np.frombuffer(b"".join(parts), np.uint8).copy()
    offs = np.zeros(len(parts) + 1, np.uint64)
    offs[1:] = np.cumsum([len(p) for p in parts])
    return reads, offs


CASES = {
    # name: (reads factory, k, p, P)
    "uniform_k31_p11_P64": (lambda: rng_reads(11, 30_000, 1500, 150, 0.005), 31, 11, 64),
    "uniform_k25_p11_P512": (lambda: rng_reads(12, 20_000, 1000, 150, 0.003), 25, 11, 512),
    "short_k10_p5_P7": (lambda: rng_reads(13, 5_000, 600, (10, 120), 0.01), 10, 5, 7),
    "edge_k25_p11_P31": (lambda: edge_reads(14), 25, 11, 31),
    "edge_k31_p11_P1": (lambda: edge_reads(15), 31, 11, 1),
    "lowcomp_k31_p11_P512": (lambda: rng_reads(16, 8_000, 800, (31, 400), 0.002, alphabet=b"AAAAAAACGTAT"), 31, 11, 512),
    "k32_p16_P97": (lambda: rng_reads(17, 10_000, 500, 150, 0.004), 32, 16, 97),
    # k > 32: the reference's LONGERKMER build
    "wide_k45_p11_P64": (lambda: rng_reads(18, 20_000, 1000, (40, 300), 0.004), 45, 11, 64),
    "wide_k63_p9_P31": (lambda: rng_reads(19, 15_000, 600, 150, 0.003), 63, 9, 31),
    "wide_k64_p16_P7": (lambda: rng_reads(20, 10_000, 400, (60, 200), 0.003), 64, 16, 7),
    "wide_edge_k33_p5_P13": (lambda: edge_reads(21), 33, 5, 13),
}


def table_order(km):
    """Ascending order of a k-mer table: u64 keys, or (low, high) pairs."""
    if km.ndim == 2:
        return np.lexsort((km[:, 0], km[:, 1]))
    return np.argsort(km, kind="stable")


def main(names):
    refs = {False: RefOracle(), True: RefOracle(wide=True)}
    if not names:
        read = b"AAAAAAAAACCCCCCCAAAAAAATGA"
        offs, mm = refs[False].gen_skm_offs(read, 10, 5)
        with open(os.path.join(HERE, "skm_test_vector.json"), "w") as f:
            json.dump({"read": read.decode(), "k": 10, "p": 5, "offsets": offs.tolist(),
                       "minimizers": mm.tolist(), "source": "cpu_funcs.cpp:654-676 (TEST main)"}, f, indent=1)
    for name, (make, k, p, P) in CASES.items():
        if names and name not in names:
            continue
        ref = refs[k > 32]
        reads, offs = make()
        pb, ps, pk, parts = ref.phase1(reads, offs, k, p, P)
        digests = [partition_digest(s) for s in parts]
        km, ct, dist, _ = ref.count_reads(reads, offs, k, p, P)
        order = table_order(km)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), reads=reads, offs=offs, k=k, p=p, P=P,
                            part_bytes=pb, part_skms=ps, part_kmers=pk, digests=np.array(digests),
                            kmers=km[order], counts=ct[order], n_distinct=dist)
        print(f"{name}: reads={len(offs) - 1} kmers={int(pk.sum())} distinct={dist} "
              f"bytes={int(pb.sum())} file={os.path.getsize(os.path.join(HERE, name + '.npz'))}")


if __name__ == "__main__":
    main(sys.argv[1:])
