"""Homopolymer compression (opt.hpc, the reference's -hpc): reads counted
with compression on give the oracle's table of the compressed reads, for
device and host input, many batches, both counters and text input."""
import numpy as np
import pytest

from conftest import sorted_table
from oracle.hpc_oracle import hpc
from tests_util import csr, random_reads

U32 = 0xFFFFFFFF


def test_oracle_known_answers():
    r, o = csr([b"AAACCGTTTT", b"", b"A", b"aAaa", b"TTTT", b"TGGG"])
    hr, ho = hpc(r, o)
    assert hr.tobytes() == b"ACGT" + b"A" + b"aAa" + b"T" + b"TG"
    assert ho.tolist() == [0, 4, 4, 5, 8, 9, 11]   # a read's first byte is kept even after an equal one


@pytest.mark.parametrize("k,p,P", [(31, 11, 64), (21, 9, 7)])
def test_oracle_pinned_to_the_reference_cpu_path(oracle, ref_oracle, k, p, P):
    """The reference's CPU phase 1 with HPC on (GenSuperkmerCPU,
    cpu_funcs.cpp:253-275) counts each compressed read without its last base:
    its _hpc_encoding returns the last index, not the length
    (cpu_funcs.cpp:92-100).  Its GPU path (GPU_HPCEncoding,
    gpu_skmgen.cu:145-173), which the B200 path follows, keeps that base.
    So the reference CPU table is the oracle's table of the compressed reads
    with each read's last byte dropped."""
    reads, offs = random_reads(31, 30_000, 800, (120, 300), 0.01)
    hr, ho = hpc(reads, offs)
    assert np.diff(ho.astype(np.int64)).min() > k  # the reference reads past shorter reads
    keep = np.ones(len(hr), bool)
    keep[ho[1:].astype(np.int64) - 1] = False
    short_r = hr[keep]
    short_o = (ho.astype(np.int64) - np.arange(len(ho))).astype(np.uint64)
    ka, ca, da, pka = ref_oracle.count_reads(reads, offs, k, p, P, 1, hpc=True)
    kb, cb, db, pkb = oracle.count_reads(short_r, short_o, k, p, P, 1)
    assert da == db and np.array_equal(pka, pkb)
    assert np.array_equal(ka, kb) and np.array_equal(ca, cb)
    assert oracle.count_reads(hr, ho, k, p, P, 1)[2] != da  # the dropped bases matter


def _reads_with_runs(seed):
    r = np.random.default_rng(seed)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    parts = []
    for _ in range(3000):
        s = acgt[r.integers(0, 4, int(r.integers(0, 300)))]
        s = np.repeat(s, r.integers(1, 5, len(s)))          # runs of 1-4
        parts.append(s.tobytes())
    parts[7] = b"A" * 20_000 + parts[7]                     # a run across tiles
    parts[8] = b"A" * 5000                                  # a read that is one run
    return csr(parts)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_hpc_counts_match_oracle(oracle, kind):
    import torch
    from rapidgkc_b200 import KmerCounter
    reads, offs = _reads_with_runs(71)
    hr, ho = hpc(reads, offs)
    k, p, P = 25, 11, 64
    ko, co, do, pko = oracle.count_reads(hr, ho, k, p, P)
    ko, co = sorted_table(ko, co)
    runs = [("device", dict()), ("host", dict(batch_bases=50_000)), ("device", dict(batch_bases=50_000)),
            ("host", dict(spill_host=True, batch_bases=50_000))]
    for src, kw in runs:
        with KmerCounter(k=k, p=p, partitions=P, counter=kind, hpc=True, **kw) as c:
            if src == "device":
                c.add_reads(torch.from_numpy(reads).cuda(), torch.from_numpy(offs.view(np.int64)).cuda())
            else:
                c.add_reads(reads, offs)
            assert np.array_equal(c.store_stats()[2], pko), (src, kw)
            n, d = c.count()
            km, ct = sorted_table(*c.result())
        assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co), (src, kw)


@pytest.mark.gpu
def test_hpc_from_fastq_text(oracle):
    from rapidgkc_b200 import KmerCounter
    reads, offs = _reads_with_runs(72)
    seqs = [reads[int(offs[i]):int(offs[i + 1])].tobytes() for i in range(len(offs) - 1)]
    text = b"".join(b"@r\n" + s + b"\n+\n" + b"I" * len(s) + b"\n" for s in seqs)
    hr, ho = hpc(reads, offs)
    k, p, P = 31, 11, 32
    ko, co, do, _ = oracle.count_reads(hr, ho, k, p, P, 2, U32)
    ko, co = sorted_table(ko, co)
    with KmerCounter(k=k, p=p, partitions=P, hpc=True) as c:
        c.add_fastx(text, "fastq")
        n, d = c.count(2, U32)
        km, ct = sorted_table(*c.result())
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)
