"""k-mers of 33 to 64 bases: the reference's 128-bit LONGERKMER build
(types.h:34-35, k <= 64 at utilities.hpp:280-281).  The CUDA path (through the
C ABI) against the oracle, whose 128-bit functions are pinned to the compiled
LONGERKMER reference by the golden fixtures wide_*.npz and by
test_oracle.py.  k-mers are (n, 2) u64 (low, high) arrays; every comparison is
bit-exact."""
import numpy as np
import pytest

from conftest import partition_digest, sorted_table
from tests_util import csr, random_reads

pytestmark = pytest.mark.gpu
U32 = 0xFFFFFFFF


def counter(k, p, P, kind="sort", **kw):
    from rapidgkc_b200 import KmerCounter
    return KmerCounter(k=k, p=p, partitions=P, counter=kind, **kw)


# windows w = k - p + 1 from 18 (four doubling levels) to 62 (three chunks)
@pytest.mark.parametrize("k,p,P,seed", [(33, 16, 64, 1), (33, 11, 512, 2), (40, 9, 31, 3), (47, 15, 7, 4),
                                        (55, 11, 128, 5), (63, 3, 2, 6), (64, 16, 13, 7), (64, 3, 97, 8)])
def test_wide_counts_and_order_match_oracle(oracle, k, p, P, seed):
    """Partition by partition, ascending 128-bit k-mers within; superkmer
    bytes equal to the oracle's in every partition."""
    reads, offs = random_reads(seed, 30_000, 1200, (k - 2, 400), 0.01)
    pbo, pso, pko, po, stream = oracle.skmgen(reads, offs, k, p, P)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    assert ko.ndim == 2
    with counter(k, p, P) as c:
        c.add_reads(reads, offs)
        pb, ps, pk = c.store_stats()
        assert np.array_equal(pb, pbo) and np.array_equal(ps, pso) and np.array_equal(pk, pko)
        for i in range(P):
            assert partition_digest(c.store_export(i)) == partition_digest(stream[int(po[i]):int(po[i + 1])])
        n, d = c.count(2, U32)
        km, ct = c.result()
    assert km.shape == (n, 2)
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


@pytest.mark.parametrize("k,p", [(45, 11), (64, 11)])
def test_wide_long_and_low_complexity_reads(oracle, k, p):
    """Superkmers past the tile's staged halo (poly-A, (AT)n) take the
    global-memory continuation; reads of k-1, k and k+1 bases; N bases."""
    r = np.random.default_rng(11)
    rnd = lambda n: bytes(np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, n)])
    parts = [rnd(20_000), b"A" * 6000, rnd(100) + b"A" * 3000 + rnd(100), b"AT" * 2500,
             rnd(k), rnd(k - 1), rnd(k + 1), b"", rnd(2047), rnd(8193), b"CAG" * 1000 + rnd(3000),
             b"ACGTNACGTN" * 40, rnd(300).lower()]
    reads, offs = csr(parts)
    P = 29
    pbo, pso, pko, po, stream = oracle.skmgen(reads, offs, k, p, P)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P) as c:
        c.add_reads(reads, offs)
        pb, ps, pk = c.store_stats()
        assert np.array_equal(pb, pbo) and np.array_equal(ps, pso) and np.array_equal(pk, pko)
        for i in range(P):
            assert partition_digest(c.store_export(i)) == partition_digest(stream[int(po[i]):int(po[i + 1])])
        n, d = c.count()
        km, ct = sorted_table(*c.result())
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


def test_wide_device_input_batches_spill_and_learned_order(oracle):
    """Device input cut into many batches, a spilled store, and a learned
    order all give the default order's table; so does the 128-bit hash
    counter, and the sort counter that a spilled store falls back to."""
    import torch
    k, p, P = 51, 11, 64
    reads, offs = random_reads(12, 40_000, 2500, (40, 600), 0.005)
    ko, co, do, pko = oracle.count_reads(reads, offs, k, p, P, 1, U32)
    ko, co = sorted_table(ko, co)
    lut = np.random.default_rng(13).permutation(4 ** p).astype(np.uint32)
    pbl, psl, pkl, _, _ = oracle.skmgen(reads, offs, k, p, P, lut)
    runs = [dict(batch_bases=20_000), dict(batch_bases=50_000, spill_host=True), dict(kind="hash"),
            dict(kind="hash", batch_bases=50_000, spill_host=True),
            dict(order=True), dict(group_keys=5000), dict(sort_seg_max=1000), dict(radix_bits=8)]
    for kw in runs:
        order = kw.pop("order", False)
        with counter(k, p, P, **kw) as c:
            if order:
                c.set_order(lut)
            c.add_reads(torch.from_numpy(reads).cuda(), torch.from_numpy(offs.view(np.int64)).cuda())
            pb, ps, pk = c.store_stats()
            if order:
                assert np.array_equal(pb, pbl) and np.array_equal(ps, psl) and np.array_equal(pk, pkl)
            else:
                assert np.array_equal(pk, pko)
            n, d = c.count()
            km, ct = sorted_table(*c.result())
        assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co), kw


def test_wide_count_reads_into_buffers_and_keys(oracle):
    """gkc_count_reads into caller buffers of two words per k-mer, host and
    device; gkc_count_keys on the same context gives one word per key."""
    import torch
    k, p, P = 60, 13, 16
    reads, offs = random_reads(14, 20_000, 800, 150, 0.003)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    with counter(k, p, P) as c:
        hk = np.zeros((len(ko) + 5, 2), np.uint64)
        hc = np.zeros(len(ko) + 5, np.uint32)
        n, d = c.count_reads(reads, offs, 2, U32, hk, hc)
        assert n == len(ko) and d == do
        assert np.array_equal(hk[:n], ko) and np.array_equal(hc[:n], co)
        dk = torch.zeros((len(ko), 2), dtype=torch.int64, device="cuda")
        dc = torch.zeros(len(ko), dtype=torch.int32, device="cuda")
        n, d = c.count_reads(reads, offs, 2, U32, dk, dc)
        assert np.array_equal(dk.cpu().numpy().view(np.uint64), ko)
        assert np.array_equal(dc.cpu().numpy().view(np.uint32), co)
        keys = np.array([7, 3, 7, 7, 1], np.uint64)
        n, d = c.count_keys(keys)
        km, ct = sorted_table(*c.result())
        assert km.ndim == 1 and km.tolist() == [1, 3, 7] and ct.tolist() == [1, 1, 3]


def test_wide_reads_shorter_than_k():
    reads, offs = csr([b"ACGT" * 10, b"", b"A" * 63])
    with counter(64, 11, 8) as c:
        assert c.count_reads(reads, offs) == (0, 0)
        assert c.result()[0].shape == (0, 2)
    seq = b"ACGTTGCAACGTTGCAACGTTGCAACGTTGCAACGTTGCAACGTTGCAACGTTGCAACGTTGCA"  # 64 bases
    reads, offs = csr([seq, seq])
    with counter(64, 11, 8) as c:
        n, d = c.count_reads(reads, offs)
        km, ct = c.result()
        assert (n, d) == (1, 1) and ct.tolist() == [2]
        v = 0
        for x in seq:
            v = (v << 2) | b"ACGT".index(x)
        rc = 0
        for x in seq[::-1]:
            rc = (rc << 2) | (3 - b"ACGT".index(x))
        m = min(v, rc)
        assert int(km[0, 0]) == m & (2**64 - 1) and int(km[0, 1]) == m >> 64
