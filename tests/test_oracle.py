"""The oracle pinned against the reference: its own known answer, the golden
fixtures produced by the reference's CPU path, and (where the reference tree
was built here) the compiled reference itself on fresh seeded inputs."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases, load_golden, partition_digest, sorted_table


def test_reference_known_answer(oracle):
    v = json.load(open(os.path.join(GOLDEN, "skm_test_vector.json")))
    offs, mm = oracle.skm_split(v["read"].encode(), v["k"], v["p"])
    assert offs.tolist() == v["offsets"] == [0, 1, 2, 8, 9, 14, 16, 17]
    assert mm.tolist() == v["minimizers"] == [767, 703, 21, 85, 336, 255, 56]


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_matches_golden(oracle, case):
    g = load_golden(case)
    k, p, P = int(g["k"]), int(g["p"]), int(g["P"])
    pb, ps, pk, po, stream = oracle.skmgen(g["reads"], g["offs"], k, p, P)
    assert np.array_equal(pb, g["part_bytes"])
    assert np.array_equal(ps, g["part_skms"])
    assert np.array_equal(pk, g["part_kmers"])
    for i in range(P):
        assert partition_digest(stream[int(po[i]):int(po[i + 1])]) == str(g["digests"][i]), f"partition {i}"
    km, ct, dist, _ = oracle.count_reads(g["reads"], g["offs"], k, p, P)
    km, ct = sorted_table(km, ct)
    assert dist == int(g["n_distinct"])
    assert np.array_equal(km, g["kmers"]) and np.array_equal(ct, g["counts"])


def test_oracle_threshold_and_saturation(oracle):
    keys = np.array([5, 5, 5, 7, 9, 9, 1, 1, 1, 1], np.uint64)
    km, ct, d = oracle.count(keys, 2, 3)
    assert d == 4 and km.tolist() == [5, 9] and ct.tolist() == [3, 2]
    km, ct, d = oracle.count(keys, 1, 0xFFFFFFFF)
    assert km.tolist() == [1, 5, 7, 9] and ct.tolist() == [4, 3, 1, 2]


def test_oracle_revcomp(oracle):
    # ACGT (k=4) = 0b00011011, its reverse complement is ACGT again
    assert oracle.revcomp(0b00011011, 4) == 0b00011011
    # AAAA -> TTTT
    assert oracle.revcomp(0, 4) == 0xFF
    assert oracle.revcomp(0, 32) == 0xFFFFFFFFFFFFFFFF


def test_hash_known_answer_distinct(oracle):
    """The reference hash counter's commented-out test
    (gpu_hash_counter.cu:693-708): keys i % 1234567 + 0xffffffff, 1234567 distinct."""
    n = 4_000_000
    keys = (np.arange(n, dtype=np.uint64) % np.uint64(1234567)) + np.uint64(0xFFFFFFFF)
    km, ct, d = oracle.count(keys, 2, 0xFFFFFFFF)
    assert d == 1234567 and len(km) == 1234567 and int(ct.sum()) == n


@pytest.mark.parametrize("k,p,P,seed", [(31, 11, 512, 1), (25, 11, 64, 2), (21, 7, 31, 3), (15, 9, 5, 4)])
def test_oracle_matches_compiled_reference(oracle, ref_oracle, k, p, P, seed):
    from tests_util import random_reads
    reads, offs = random_reads(seed, 20_000, 800, (k, 300), 0.01)
    a = ref_oracle.phase1(reads, offs, k, p, P)
    b = oracle.skmgen(reads, offs, k, p, P)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    po = b[3]
    for i in range(P):
        assert partition_digest(a[3][i]) == partition_digest(b[4][int(po[i]):int(po[i + 1])])
    ka, ca, da, _ = ref_oracle.count_reads(reads, offs, k, p, P, cmin=2)
    kb, cb, db, _ = oracle.count_reads(reads, offs, k, p, P, cmin=2)
    assert da == db
    assert np.array_equal(ka, kb) and np.array_equal(ca, cb)


@pytest.mark.parametrize("k,p,P,seed", [(33, 11, 64, 5), (48, 13, 31, 6), (64, 16, 7, 7), (57, 3, 5, 8)])
def test_oracle_matches_compiled_reference_wide(oracle, ref_oracle_wide, k, p, P, seed):
    """k > 32 against the reference's 128-bit LONGERKMER build (types.h:34-35)."""
    from tests_util import random_reads
    reads, offs = random_reads(seed, 20_000, 500, (k - 3, 300), 0.01)
    a = ref_oracle_wide.phase1(reads, offs, k, p, P)
    b = oracle.skmgen(reads, offs, k, p, P)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    ka, ca, da, _ = ref_oracle_wide.count_reads(reads, offs, k, p, P, cmin=2)
    kb, cb, db, _ = oracle.count_reads(reads, offs, k, p, P, cmin=2)
    assert da == db and ka.shape == kb.shape and ka.ndim == 2
    assert np.array_equal(ka, kb) and np.array_equal(ca, cb)


def test_oracle_wide_revcomp_and_order(oracle):
    """128-bit keys: a k=64 k-mer and its reverse complement share one
    canonical form, and the table is ordered by (high, low)."""
    seq = np.frombuffer(b"ACGT" * 16, np.uint8)
    # one superkmer of k=64 bases: first byte holds 3 bases (phase 0), then
    # full bytes, then a terminal byte with 64 % 3 = 1 base
    def pack(s):
        codes = {65: 0, 67: 1, 71: 2, 84: 3}
        c = [codes[x] for x in s]
        out = [0xC0 | (c[0] << 4) | (c[1] << 2) | c[2]]
        i = 3
        while len(c) - i >= 3:
            out.append(0xC0 | (c[i] << 4) | (c[i + 1] << 2) | c[i + 2])
            i += 3
        rem = len(c) - i
        last = rem << 6
        for t in range(rem):
            last |= c[i + t] << (4 - 2 * t)
        out.append(last)
        return np.array(out, np.uint8)
    a = oracle.extract(pack(bytes(seq)), 64)
    comp = bytes(b"TGCA"[b"ACGT".index(x)] for x in bytes(seq)[::-1])
    b = oracle.extract(pack(comp), 64)
    assert a.shape == (1, 2) and np.array_equal(a, b)
    # ACGT repeated is its own reverse complement: the value itself
    v = 0
    for x in bytes(seq):
        v = (v << 2) | b"ACGT".index(x)
    assert int(a[0, 0]) == v & (2**64 - 1) and int(a[0, 1]) == v >> 64
    keys = np.array([[5, 1], [9, 0], [5, 1], [0, 2]], np.uint64)
    km, ct, d = oracle.count(keys)
    assert d == 3 and km.tolist() == [[9, 0], [5, 1], [0, 2]] and ct.tolist() == [1, 2, 1]


@pytest.mark.parametrize("k,p,P,seed", [(12, 5, 7, 1), (16, 9, 31, 2), (9, 3, 3, 3)])
def test_oracle_matches_compiled_reference_short(oracle, k, p, P, seed):
    """k <= 16 against the reference's 32-bit SHORTERKMER build (types.h:36-37,
    utilities.hpp:277-278): the same k-mer values, held in u32 there."""
    import os
    from conftest import ROOT
    from oracle.oracle import RefOracle
    from tests_util import random_reads
    path = os.path.join(ROOT, "oracle", "_ref", "libgkc_ref_short.so")
    if not os.path.exists(path):
        pytest.skip(f"{path} missing")
    ref = RefOracle(path=path)
    assert ref.lib.ref_kmer_bits() == 32
    reads, offs = random_reads(seed, 20_000, 800, (k, 300), 0.01)
    ka, ca, da, pka = ref.count_reads(reads, offs, k, p, P, 2)
    kb, cb, db, pkb = oracle.count_reads(reads, offs, k, p, P, 2)
    assert da == db and np.array_equal(pka, pkb)
    assert np.array_equal(ka, kb) and np.array_equal(ca, cb)


def test_reference_digest_matches_oracle(oracle, ref_oracle):
    """The digest bench.py compares against (the reference's phase 1, its
    extraction and sort, run-length count, threshold) equals the digest of
    the C restatement's table, on a sample of the skewed workload."""
    from rapidgkc_b200 import synth
    reads, offs = synth.make_workload("skewed_200m", scale=0.001, threads=4)
    for k, cmin in ((31, 2), (25, 1)):
        d = ref_oracle.digest(reads, offs, k, 11, 64, threads=4, cmin=cmin)
        km, ct, dist, pk = oracle.count_reads(reads, offs, k, 11, 64, cmin)
        assert d["kept"] == len(km) and d["distinct"] == dist and d["instances"] == int(pk.sum())
        assert d["xor"] == int(np.bitwise_xor.reduce(km))
        assert d["sum_kc"] == int(np.sum(km * ct.astype(np.uint64), dtype=np.uint64))
        assert d["sum_c"] == int(ct.sum(dtype=np.uint64))
