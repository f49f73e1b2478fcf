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
