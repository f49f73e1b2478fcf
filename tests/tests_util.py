"""Seeded small inputs for tests (numpy only; no GPU)."""
import numpy as np


def random_reads(seed, genome_len, n_reads, read_len, err, alphabet=b"ACGT", both_strands=True):
    r = np.random.default_rng(seed)
    g = np.frombuffer(alphabet, np.uint8)[r.integers(0, len(alphabet), genome_len)]
    comp = np.zeros(256, np.uint8)
    for a, b in zip(b"ACGTNacgtn", b"TGCANtgcan"):
        comp[a] = b
    reads, offs = [], [0]
    for _ in range(n_reads):
        if np.isscalar(read_len):
            L = int(read_len)
        else:
            L = int(r.integers(read_len[0], read_len[1] + 1))
        L = min(L, genome_len)
        pos = int(r.integers(0, genome_len - L + 1))
        s = g[pos:pos + L].copy()
        if both_strands and r.integers(0, 2):
            s = comp[s[::-1]]
        m = r.random(L) < err
        s[m] = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, int(m.sum()))]
        reads.append(s)
        offs.append(offs[-1] + L)
    reads = np.concatenate(reads).astype(np.uint8) if reads else np.zeros(0, np.uint8)
    return reads, np.array(offs, np.uint64)


def csr(parts):
    reads = np.frombuffer(b"".join(parts), np.uint8).copy()
    offs = np.zeros(len(parts) + 1, np.uint64)
    offs[1:] = np.cumsum([len(p) for p in parts])
    return reads, offs
