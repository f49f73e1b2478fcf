"""gkc_main, the command-line counter: argument handling (CPU) and its output
against the oracle on FASTQ / gzip FASTA input (GPU)."""
import gzip
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, sorted_table
from tests_util import random_reads

CLI = os.path.join(ROOT, "rapidgkc_b200", "gkc_main")
U32 = 0xFFFFFFFF


def _run(*args, check=True):
    p = subprocess.run([CLI, *args], capture_output=True, text=True, timeout=600)
    if check and p.returncode != 0:
        raise AssertionError(f"gkc_main {' '.join(args)} -> {p.returncode}\n{p.stderr}")
    return p


@pytest.mark.parametrize("args,msg", [([], "no input"), (["-cpuonly", "-read", "x.fq"], "no CPU path"),
                                      (["-of", "csv", "-read", "x.fq"], "-of must be"),
                                      (["-ngpu", "2", "-read", "x.fq"], "one GPU"),
                                      (["-ci", "5", "-cx", "2", "-read", "x.fq"], "larger than")])
def test_cli_rejects_bad_arguments(args, msg):
    p = _run(*args, check=False)
    assert p.returncode == 2 and msg in p.stderr


def test_cli_rejects_k_beyond_64(tmp_path):
    """k up to 64 is accepted (the reference's 128-bit build); 65 is refused
    by the library before any device call."""
    fq = tmp_path / "x.fq"
    fq.write_bytes(b"@r\nACGT\n+\nIIII\n")
    p = _run("-k", "65", "-p", "11", "-skm", "16", "-read", str(fq), check=False)
    assert p.returncode == 1 and "invalid argument" in p.stderr


def _write_inputs(tmp, reads, offs):
    seqs = [reads[int(offs[i]):int(offs[i + 1])].tobytes() for i in range(len(offs) - 1)]
    h = len(seqs) // 2
    fq = os.path.join(tmp, "a.fq")
    with open(fq, "wb") as f:
        for i, s in enumerate(seqs[:h]):
            f.write(b"@r%d\n%s\n+\n%s\n" % (i, s, b"I" * len(s)))
    fa = os.path.join(tmp, "b.fa.gz")
    with gzip.open(fa, "wb") as f:
        for i, s in enumerate(seqs[h:]):
            f.write(b">r%d description\n" % i)
            for j in range(0, len(s), 60):  # multi-line FASTA, with a CRLF line
                f.write(s[j:j + 60] + (b"\r\n" if j == 0 else b"\n"))
    return fq, fa


def _read_bin(path):
    b = open(path, "rb").read()
    assert b[:8] == b"GKCB1\0\0\0"
    k, _, n = np.frombuffer(b[8:24], np.uint32)[0], 0, int(np.frombuffer(b[16:24], np.uint64)[0])
    rec = np.frombuffer(b[24:], dtype=np.dtype([("k", "<u8"), ("c", "<u4")]), count=n)
    return int(k), rec["k"].copy(), rec["c"].copy()


@pytest.mark.gpu
def test_cli_counts_match_oracle(oracle, tmp_path):
    k, p, P = 25, 11, 32
    reads, offs = random_reads(91, 30_000, 4000, (60, 400), 0.005)
    fq, fa = _write_inputs(str(tmp_path), reads, offs)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    ko, co = sorted_table(ko, co)
    out = str(tmp_path / "counts.bin")
    p_ = _run("-k", str(k), "-p", str(p), "-skm", str(P), "-ci", "2", "-o", out, "-sorted", "-t", "8",
              "-read", fq, fa)
    assert f"distinct k-mers {do}" in p_.stderr
    # the reference's own report lines (gkc_main.cpp:385, 433)
    assert f"Total number of distinct kmers: {do}" in p_.stderr
    assert float(p_.stdout.strip().splitlines()[-1]) > 0
    kk, km, ct = _read_bin(out)
    assert kk == k and np.all(np.diff(km.astype(np.int64)) > 0)
    assert np.array_equal(km, ko) and np.array_equal(ct, co)
    # text output, sort counter, learned order: the same multiset
    out2 = str(tmp_path / "counts.txt")
    _run("-k", str(k), "-p", str(p), "-skm", str(P), "-ci", "2", "-o", out2, "-of", "txt", "-counter", "sort",
         "-order", "learned", "-bb", "1", "-read", fq, fa)
    lines = open(out2).read().split()
    code = {"A": 0, "C": 1, "G": 2, "T": 3}
    km2 = np.array([int("".join(str(code[ch]) for ch in s), 4) for s in lines[0::2]], np.uint64)
    ct2 = np.array(lines[1::2], np.uint32)
    km2, ct2 = sorted_table(km2, ct2)
    assert np.array_equal(km2, ko) and np.array_equal(ct2, co)


@pytest.mark.gpu
def test_cli_fasta_records_longer_than_a_block(oracle, tmp_path):
    """-bb 1 reads 1 MB blocks: a 2.5 Mbp FASTA record (wrapped at 80) is cut
    inside twice, and the k-1 bases repeated across each cut keep its k-mers
    exact; short records around it stay whole."""
    r = np.random.default_rng(5)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    big = bytes(acgt[r.integers(0, 4, 2_500_000)])
    small = [bytes(acgt[r.integers(0, 4, int(n))]) for n in r.integers(40, 400, 50)]
    seqs = small[:25] + [big] + small[25:]
    path = str(tmp_path / "g.fa")
    with open(path, "wb") as f:
        for i, s in enumerate(seqs):
            f.write(b">s%d\n" % i + b"\n".join(s[j:j + 80] for j in range(0, len(s), 80)) + b"\n")
    reads = np.frombuffer(b"".join(seqs), np.uint8).copy()
    offs = np.zeros(len(seqs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in seqs])
    k, p, P = 31, 11, 64
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 1, U32)
    ko, co = sorted_table(ko, co)
    out = str(tmp_path / "c.bin")
    p_ = _run("-k", str(k), "-p", str(p), "-skm", str(P), "-ci", "1", "-o", out, "-sorted", "-bb", "1", "-read", path)
    assert f"distinct k-mers {do}" in p_.stderr and f"bases {len(reads)}," in p_.stderr
    _, km, ct = _read_bin(out)
    assert np.array_equal(km, ko) and np.array_equal(ct, co)


@pytest.mark.gpu
def test_cli_wide_kmers(oracle, tmp_path):
    """k = 47 (the reference's 128-bit build): binary records of low word,
    high word and count, sorted as 128-bit values; text k-mers of 47 bases."""
    k, p, P = 47, 11, 16
    reads, offs = random_reads(92, 20_000, 1500, (50, 300), 0.005)
    fq, fa = _write_inputs(str(tmp_path), reads, offs)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    ko, co = sorted_table(ko, co)
    out = str(tmp_path / "wide.bin")
    p_ = _run("-k", str(k), "-p", str(p), "-skm", str(P), "-ci", "2", "-o", out, "-sorted", "-read", fq, fa)
    assert f"distinct k-mers {do}" in p_.stderr
    b = open(out, "rb").read()
    assert b[:8] == b"GKCB1\0\0\0" and int(np.frombuffer(b[8:12], np.uint32)[0]) == k
    n = int(np.frombuffer(b[16:24], np.uint64)[0])
    rec = np.frombuffer(b[24:], dtype=np.dtype([("lo", "<u8"), ("hi", "<u8"), ("c", "<u4")]), count=n)
    km = np.stack([rec["lo"], rec["hi"]], axis=1)
    assert np.array_equal(km, ko) and np.array_equal(rec["c"], co)
    out2 = str(tmp_path / "wide.txt")
    _run("-k", str(k), "-p", str(p), "-skm", str(P), "-ci", "2", "-o", out2, "-of", "txt", "-read", fq, fa)
    lines = open(out2).read().split()
    code = {"A": 0, "C": 1, "G": 2, "T": 3}
    vals = [int("".join(str(code[ch]) for ch in s), 4) for s in lines[0::2]]
    assert all(len(s) == k for s in lines[0::2])
    km2 = np.array([[v & (2**64 - 1), v >> 64] for v in vals], np.uint64)
    km2, ct2 = sorted_table(km2, np.array(lines[1::2], np.uint32))
    assert np.array_equal(km2, ko) and np.array_equal(ct2, co)


@pytest.mark.gpu
def test_cli_reference_defaults(oracle, tmp_path):
    """No -k / -p / -skm: the reference's defaults (k=21, p=7, 31 partitions,
    utilities.hpp:187-189) and its report lines."""
    reads, offs = random_reads(93, 8_000, 2000, (40, 300), 0.005)
    fq, fa = _write_inputs(str(tmp_path), reads, offs)  # half the reads in each file
    ko, co, do, pk = oracle.count_reads(reads, offs, 21, 7, 31, 1, U32)
    out = str(tmp_path / "counts.bin")
    p_ = _run("-o", out, "-sorted", "-read", fq, fa)
    assert f"Total number of distinct kmers: {do}" in p_.stderr
    assert f"KMER TOT CNT = {int(pk.sum())}" in p_.stderr
    kk, km, ct = _read_bin(out)
    ko, co = sorted_table(ko, co)
    assert kk == 21 and np.array_equal(km, ko) and np.array_equal(ct, co)
