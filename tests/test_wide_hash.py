"""The sub-bucket hash counter for k-mers of 33 to 64 bases (u128 keys,
count_wide.cu) against the oracle, whose 128-bit functions are pinned to the
reference's compiled LONGERKMER build.  The hash counter's output is not
ordered, so tables are compared sorted; every comparison is bit-exact."""
import numpy as np
import pytest

from conftest import sorted_table
from tests_util import csr, random_reads

pytestmark = pytest.mark.gpu
U32 = 0xFFFFFFFF


def counter(k, p, P, **kw):
    from rapidgkc_b200 import KmerCounter
    return KmerCounter(k=k, p=p, partitions=P, counter="hash", **kw)


@pytest.mark.parametrize("k,p,P,seed,cmin", [(33, 16, 64, 1, 2), (47, 15, 7, 4, 1), (63, 11, 128, 5, 2),
                                             (64, 16, 13, 7, 1), (40, 9, 31, 3, 3)])
def test_wide_hash_matches_oracle(oracle, k, p, P, seed, cmin):
    reads, offs = random_reads(seed, 30_000, 1200, (k - 2, 400), 0.01)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, cmin, U32)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P) as c:
        n, d = c.count_reads(reads, offs, cmin, U32)
        km, ct = sorted_table(*c.result())
    assert km.shape == (n, 2)
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


@pytest.mark.parametrize("k,p", [(45, 11), (64, 11)])
def test_wide_hash_low_complexity_takes_the_sort(oracle, k, p):
    """A poly-A read of 1.1 Mbp makes a sub-bucket of more than 2^20
    instances: it is extracted and counted by the 128-bit radix sort, beside
    the hash counter's own sub-buckets; (AT)n and (CAG)n runs make heavy
    sub-buckets that are counted in pieces."""
    r = np.random.default_rng(11)
    rnd = lambda n: bytes(np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, n)])
    parts = [rnd(20_000), b"A" * 1_100_000, rnd(100) + b"A" * 3000 + rnd(100), b"AT" * 25_000,
             rnd(k), rnd(k - 1), rnd(k + 1), b"", rnd(2047), rnd(8193), b"CAG" * 1000 + rnd(3000),
             b"ACGTNACGTN" * 40, rnd(300).lower()]
    reads, offs = csr(parts)
    P = 29
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P) as c:
        n, d = c.count_reads(reads, offs)
        km, ct = sorted_table(*c.result())
        t = c.timings()
    assert t["overflowed_sub_buckets"] >= 1
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


@pytest.mark.parametrize("n_x,route", [(150, "one"), (600, "split"), (6000, "sort")])
def test_wide_hash_overflowing_sub_bucket(oracle, n_x, route):
    """A minimizer X made the preferred one for n_x reads of 150 bases: each
    read adds the 35 k-mers that contain X to X's sub-bucket, all distinct.
    150 reads (5k keys) overflow the 4096-slot table and fit the second
    pass's 8192; 600 (21k) are counted in two key-hash pieces that overflow
    and split into four; 6000 (210k) in pieces whose split would decode more
    than the limit, so those pieces go to the radix sort, with the key filter.
    Every route gives the oracle's multiset."""
    k, p, P = 45, 11, 4
    r = np.random.default_rng(41)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    rnd = lambda n: bytes(acgt[r.integers(0, 4, n)])
    X = b"CTTGACCGTAG"
    parts = [rnd(70) + X + rnd(69) for _ in range(n_x)] + [rnd(150) for _ in range(3000)]
    reads, offs = csr(parts)
    code = lambda s: int("".join(str("ACGT".index(chr(ch))) for ch in s), 4)
    lut = r.permutation(4 ** p).astype(np.uint32)
    j = int(np.nonzero(lut == 0)[0][0])
    lut[j], lut[code(X)] = lut[code(X)], 0
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P) as c:
        c.set_order(lut)
        n, d = c.count_reads(reads, offs)
        km, ct = sorted_table(*c.result())
        t = c.timings()
    if route == "one":
        assert t["second_pass_sub_buckets"] >= 1 and t["overflowed_sub_buckets"] == 0
    elif route == "split":
        assert t["second_pass_sub_buckets"] >= 4 and t["overflowed_sub_buckets"] == 0
    else:
        assert t["overflowed_sub_buckets"] >= 2
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


def test_wide_hash_host_buffers_and_partition_subsets(oracle):
    """gkc_count_reads into host buffers of two words per k-mer, and
    gkc_count_partitions over two disjoint subsets adding up to the whole."""
    k, p, P = 60, 13, 16
    reads, offs = random_reads(14, 20_000, 800, 150, 0.003)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P) as c:
        hk = np.zeros((len(ko) + 5, 2), np.uint64)
        hc = np.zeros(len(ko) + 5, np.uint32)
        n, d = c.count_reads(reads, offs, 2, U32, hk, hc)
        assert n == len(ko) and d == do
        km, ct = sorted_table(hk[:n], hc[:n])
        assert np.array_equal(km, ko) and np.array_equal(ct, co)
        tabs, dist = [], 0
        c.add_reads(reads, offs)
        for parts in (range(0, P, 2), range(1, P, 2)):
            n1, d1 = c.count_partitions(list(parts), 2, U32)
            tabs.append(c.result())
            dist += d1
        km = np.concatenate([t[0] for t in tabs])
        ct = np.concatenate([t[1] for t in tabs])
        km, ct = sorted_table(km, ct)
    assert dist == do and np.array_equal(km, ko) and np.array_equal(ct, co)
