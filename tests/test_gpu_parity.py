"""Parity of the CUDA path (through the C ABI) with the reference's outputs:
golden fixtures made by the reference's own CPU path, and the oracle on fresh
seeded inputs.  Integer work: every comparison is bit-exact."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden, partition_digest, sorted_table
from tests_util import csr, random_reads

pytestmark = pytest.mark.gpu
U32 = 0xFFFFFFFF


def counter(k, p, P, kind="hash", **kw):
    from rapidgkc_b200 import KmerCounter
    return KmerCounter(k=k, p=p, partitions=P, counter=kind, **kw)


@pytest.mark.parametrize("case", golden_cases())
def test_golden_superkmers(case):
    g = load_golden(case)
    k, p, P = int(g["k"]), int(g["p"]), int(g["P"])
    with counter(k, p, P) as c:
        c.add_reads(g["reads"], g["offs"])
        pb, ps, pk = c.store_stats()
        assert np.array_equal(pb, g["part_bytes"])
        assert np.array_equal(ps, g["part_skms"])
        assert np.array_equal(pk, g["part_kmers"])
        for i in range(P):
            assert partition_digest(c.store_export(i)) == str(g["digests"][i]), f"partition {i}"


@pytest.mark.parametrize("kind", ["hash", "sort"])
@pytest.mark.parametrize("case", golden_cases())
def test_golden_counts(case, kind):
    g = load_golden(case)
    k, p, P = int(g["k"]), int(g["p"]), int(g["P"])
    with counter(k, p, P, kind) as c:
        c.add_reads(g["reads"], g["offs"])
        n, d = c.count(1, U32)
        km, ct = sorted_table(*c.result())
        assert d == int(g["n_distinct"]) and n == len(g["kmers"])
        assert np.array_equal(km, g["kmers"]) and np.array_equal(ct, g["counts"])
        # threshold [2, 5] on the same input
        c.add_reads(g["reads"], g["offs"])
        n, d = c.count(2, 5)
        km, ct = sorted_table(*c.result())
        keep = (g["counts"] >= 2) & (g["counts"] <= 5)
        assert d == int(g["n_distinct"])
        assert np.array_equal(km, g["kmers"][keep]) and np.array_equal(ct, g["counts"][keep])


@pytest.mark.parametrize("k,p,P,seed", [(31, 11, 512, 1), (25, 11, 64, 2), (21, 7, 31, 3), (15, 9, 5, 4),
                                        (32, 16, 4096, 5), (12, 3, 2, 6)])
def test_sort_counter_order_matches_oracle(oracle, k, p, P, seed):
    """The sort counter emits partition by partition, ascending within."""
    reads, offs = random_reads(seed, 30_000, 1200, (k, 260), 0.01)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    with counter(k, p, P, "sort") as c:
        n, d = c.count_reads(reads, offs, 2, U32)
        km, ct = c.result()
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_device_input_and_many_batches(oracle, kind):
    import torch
    reads, offs = random_reads(7, 50_000, 4000, (20, 400), 0.005)
    k, p, P = 27, 10, 128
    ko, co, do, pko = oracle.count_reads(reads, offs, k, p, P)
    ko, co = sorted_table(ko, co)
    # device input
    with counter(k, p, P, kind) as c:
        dr = torch.from_numpy(reads).cuda()
        do_ = torch.from_numpy(offs.view(np.int64)).cuda()
        c.add_reads(dr, do_)
        assert np.array_equal(c.store_stats()[2], pko)
        n, d = c.count()
        km, ct = sorted_table(*c.result())
        assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)
    # device input in place, in many small batches (batch_cuts_kernel)
    with counter(k, p, P, kind, batch_bases=30_000) as c:
        dr = torch.from_numpy(reads).cuda()
        do_ = torch.from_numpy(offs.view(np.int64)).cuda()
        c.add_reads(dr, do_)
        assert len(c.batch_timings()) >= int(offs[-1]) // 30_000 - 1
        assert np.array_equal(c.store_stats()[2], pko)
        n, d = c.count()
        km, ct = sorted_table(*c.result())
        assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)
    # host input split into many small batches, added in two calls
    with counter(k, p, P, kind, batch_bases=30_000) as c:
        h = len(offs) // 2
        c.add_reads(reads, offs[: h + 1])
        c.add_reads(reads[int(offs[h]):], offs[h:] - offs[h])
        assert np.array_equal(c.store_stats()[2], pko)
        n, d = c.count()
        km, ct = sorted_table(*c.result())
        assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_long_and_low_complexity_reads(oracle, kind):
    """Superkmers longer than a tile's halo (poly-A, (AT)n) and reads spanning
    many tiles take the kernel's global-memory continuation path."""
    r = np.random.default_rng(8)
    rnd = lambda n: bytes(np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, n)])
    parts = [rnd(20_000), b"A" * 6000, rnd(100) + b"A" * 3000 + rnd(100), b"AT" * 2500,
             rnd(31), rnd(30), b"", rnd(2047), rnd(2048), rnd(2049), b"CAG" * 1000 + rnd(3000)]
    reads, offs = csr(parts)
    for k, p, P in [(31, 11, 64), (25, 11, 7)]:
        pbo, pso, pko, po, stream = oracle.skmgen(reads, offs, k, p, P)
        ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P)
        ko, co = sorted_table(ko, co)
        with counter(k, p, P, kind) as c:
            c.add_reads(reads, offs)
            pb, ps, pk = c.store_stats()
            assert np.array_equal(pb, pbo) and np.array_equal(ps, pso) and np.array_equal(pk, pko)
            for i in range(P):
                assert partition_digest(c.store_export(i)) == partition_digest(stream[int(po[i]):int(po[i + 1])])
            n, d = c.count()
            km, ct = sorted_table(*c.result())
            assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_device_batches_with_reads_longer_than_a_batch(oracle, kind):
    """Device input cut into batches of 1000 bases, with reads of up to 5000
    bases (a read spans several cuts) and a 20 kb poly-A read."""
    import torch
    r = np.random.default_rng(17)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    parts = [bytes(acgt[r.integers(0, 4, int(n))]) for n in r.integers(20, 5000, 400)]
    parts[100] = b"A" * 20_000
    reads, offs = csr(parts)
    k, p, P = 31, 11, 32
    ko, co, do, pko = oracle.count_reads(reads, offs, k, p, P)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P, kind, batch_bases=1000) as c:
        c.add_reads(torch.from_numpy(reads).cuda(), torch.from_numpy(offs.view(np.int64)).cuda())
        assert np.array_equal(c.store_stats()[2], pko)
        n, d = c.count()
        km, ct = sorted_table(*c.result())
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


def test_reads_shorter_than_k_and_empty():
    reads, offs = csr([b"ACGT" * 7, b"", b"A", b"ACGTACGTACGTACGTACGTACGTACGTAC"])  # all < 31
    with counter(31, 11, 16) as c:
        n, d = c.count_reads(reads, offs)
        assert (n, d) == (0, 0)
    reads, offs = csr([b"ACGTTGCAACGTTGCAACGTTGCAACGTTGC"])  # exactly k
    with counter(31, 11, 16, "sort") as c:
        n, d = c.count_reads(reads, offs)
        assert (n, d) == (1, 1)


@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_learned_order_keeps_the_multiset(oracle, kind):
    """Any minimizer order yields the same (k-mer, count) multiset; the
    partition contents follow the order (checked against the oracle)."""
    k, p, P = 31, 11, 256
    reads, offs = random_reads(9, 40_000, 3000, 150, 0.004)
    lut = np.random.default_rng(10).permutation(4 ** p).astype(np.uint32)
    k0, c0, d0, _ = oracle.count_reads(reads, offs, k, p, P)
    pbo, pso, pko, _, _ = oracle.skmgen(reads, offs, k, p, P, lut)
    with counter(k, p, P, kind) as c:
        c.set_order(lut)
        c.add_reads(reads, offs)
        pb, ps, pk = c.store_stats()
        assert np.array_equal(pb, pbo) and np.array_equal(ps, pso) and np.array_equal(pk, pko)
        n, d = c.count()
        km, ct = sorted_table(*c.result())
    k0, c0 = sorted_table(k0, c0)
    assert d == d0 and np.array_equal(km, k0) and np.array_equal(ct, c0)


@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_hash_known_answer(kind):
    """gpu_hash_counter.cu:693-708: 40M keys i % 1234567 + 0xffffffff."""
    n = 40_000_000
    keys = (np.arange(n, dtype=np.uint64) % np.uint64(1234567)) + np.uint64(0xFFFFFFFF)
    with counter(31, 11, 1, kind) as c:
        kept, d = c.count_keys(keys, 2, U32)
        assert d == 1234567 and kept == 1234567
        km, ct = sorted_table(*c.result())
        assert np.array_equal(km, np.arange(1234567, dtype=np.uint64) + np.uint64(0xFFFFFFFF))
        assert int(ct.sum()) == n and ct.min() == 32 and ct.max() == 33


@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_count_keys_matches_oracle(oracle, kind):
    r = np.random.default_rng(11)
    keys = r.integers(0, 1 << 20, 3_000_000, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    keys = keys[keys != np.uint64(0xFFFFFFFFFFFFFFFF)]
    ko, co, do = oracle.count(keys, 3, 10)
    with counter(31, 11, 1, kind) as c:
        n, d = c.count_keys(keys, 3, 10)
        km, ct = sorted_table(*c.result())
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


def test_retries_spill_and_groups(oracle):
    """Undersized hash tables are retried larger; a spilled store and small
    sort groups give the same result."""
    k, p, P = 31, 11, 64
    reads, offs = random_reads(12, 60_000, 5000, 150, 0.01)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    ko, co = sorted_table(ko, co)
    for kw, kind in [(dict(table_slots=0.02, hash_l2_only=True), "hash"), (dict(hash_l2_only=True), "hash"),
                     (dict(spill_host=True), "hash"), (dict(spill_host=True, hash_l2_only=True), "hash"),
                     (dict(spill_host=True, batch_bases=500_000), "hash"),  # many spilled chunks staged together
                     (dict(spill_host=True, batch_bases=500_000), "sort"),
                     (dict(spill_host=True, group_keys=50_000), "sort"), (dict(group_keys=1), "sort"),
                     (dict(radix_bits=5), "sort"), (dict(radix_bits=8), "sort"), (dict(radix_bits=10), "sort"),
                     # partitions above sort_seg_max keys take the three-kernel sort (some do, some not)
                     (dict(sort_seg_max=20_000), "sort"), (dict(sort_seg_max=1, radix_bits=11), "sort")]:
        with counter(k, p, P, kind, **kw) as c:
            c.add_reads(reads, offs)
            n, d = c.count(2, U32)
            km, ct = sorted_table(*c.result())
        assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co), kw


@pytest.mark.parametrize("pinned,redo", [(True, False), (False, False), (True, True)])
def test_host_output_streamed_by_groups(oracle, pinned, redo, monkeypatch):
    """count_reads into host arrays: the hash counter counts in partition
    groups of halving size (1/2, 1/4, 1/8, 1/16 of the store, then the rest)
    and copies each group's k-mers out while the next group counts (forced
    output overflows redo every group before its copy)."""
    import torch
    if redo:
        monkeypatch.setenv("GKC_OUT_ESTIMATE", "1")
    k, p, P = 31, 11, 64
    reads, offs = random_reads(15, 200_000, 20_000, 150, 0.01)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    cap = len(ko) + 100
    if pinned:
        hk = torch.zeros(cap, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
        hc = torch.zeros(cap, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    else:
        hk, hc = np.zeros(cap, np.uint64), np.zeros(cap, np.uint32)
    with counter(k, p, P, "hash") as c:
        for _ in range(2):
            n, d = c.count_reads(reads, offs, 2, U32, out_kmers=hk, out_counts=hc)
            assert c.timings()["phase2_groups"] >= 3
            km, ct = sorted_table(hk[:n].copy(), hc[:n].copy())
            assert d == do and n == len(ko)
            assert np.array_equal(km, sorted_table(ko, co)[0]) and np.array_equal(ct, sorted_table(ko, co)[1])
            rk, rc = sorted_table(*c.result())                 # the device result is the same table
            assert np.array_equal(rk, km) and np.array_equal(rc, ct)
        with pytest.raises(Exception):
            c.count_reads(reads, offs, 2, U32, out_kmers=hk[:10], out_counts=hc[:10])  # too small


@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_spill_arena_reserve_and_reuse(oracle, kind):
    """Spilled chunks take pinned memory reserved ahead (from another thread)
    and reuse it after the store is counted: the second pass pins nothing."""
    import threading
    k, p, P = 31, 11, 64
    reads, offs = random_reads(14, 60_000, 5000, 150, 0.01)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P, kind, spill_host=True, batch_bases=200_000) as c:
        th = threading.Thread(target=c.reserve_host, args=(1 << 20,))
        th.start()
        c.add_reads(reads, offs)
        th.join()
        pinned = c.reserve_host(0)
        assert pinned >= 1 << 20
        assert c.reserve_host(pinned // 2) == pinned   # already held: nothing more is pinned
        for _ in range(2):
            n, d = c.count(2, U32)
            km, ct = sorted_table(*c.result())
            assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)
            c.add_reads(reads, offs)
        assert c.reserve_host(0) == pinned


def test_shared_memory_overflow_falls_back(oracle):
    """Partitions with far more distinct k-mers than a CTA's shared-memory
    table are counted through the L2 table with the same result."""
    k, p, P = 31, 11, 2
    reads, offs = random_reads(13, 200_000, 3000, 150, 0.02)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P, "hash") as c:
        n, d = c.count_reads(reads, offs)
        km, ct = sorted_table(*c.result())
    assert d == do and d > 100_000
    assert np.array_equal(km, ko) and np.array_equal(ct, co)


@pytest.mark.parametrize("record_slice", [None, "1"])
def test_heavy_and_overflowing_sub_buckets(oracle, record_slice, monkeypatch):
    """A learned order that makes two p-mers the preferred minimizers builds
    three kinds of sub-bucket beside ordinary ones: one with ~31k distinct
    k-mers (overflows the shared-memory table), one with ~105k distinct k-mers
    (above the heavy limit, so it is never counted by one CTA), and (AT)n reads
    whose 120k k-mer instances share one or two distinct k-mers.  All take the
    record split and give the oracle's multiset; with record_slice each such
    sub-bucket is counted in a record slice of its own."""
    if record_slice:
        monkeypatch.setenv("GKC_RECORD_SLICE", record_slice)
    k, p, P = 31, 11, 4
    r = np.random.default_rng(21)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    rnd = lambda n: bytes(acgt[r.integers(0, 4, n)])
    X, Y = b"CTTGACCGTAG", b"GATCCTAGGCA"
    parts = [rnd(70) + X + rnd(69) for _ in range(1500)] + [rnd(60) + Y + rnd(79) for _ in range(5000)]
    parts += [b"AT" * 75 for _ in range(1000)] + [rnd(150) for _ in range(3000)]
    reads, offs = csr(parts)
    code = lambda s: int("".join(str("ACGT".index(chr(ch))) for ch in s), 4)
    lut = r.permutation(4 ** p).astype(np.uint32)
    for v, rank in [(code(X), 0), (code(Y), 1)]:
        j = int(np.nonzero(lut == rank)[0][0])
        lut[j], lut[v] = lut[v], rank
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P, "hash") as c:
        c.set_order(lut)
        n, d = c.count_reads(reads, offs)
        km, ct = sorted_table(*c.result())
        t = c.timings()
    assert t["overflowed_sub_buckets"] >= 2  # the (AT)n minimizer may share a sub-bucket
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


def test_second_pass_counts_a_moderately_overflowing_sub_bucket(oracle):
    """One minimizer made the preferred one for 250 reads adds ~5k distinct
    k-mers to its sub-bucket (about 4-8k instances of other minimizers):
    more than the first 8192-slot table holds, well within the second pass's
    16384 slots.  It is counted there, not by the record split, with the
    oracle's multiset."""
    k, p, P = 31, 11, 4
    r = np.random.default_rng(33)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    rnd = lambda n: bytes(acgt[r.integers(0, 4, n)])
    X = b"CTTGACCGTAG"
    parts = [rnd(70) + X + rnd(69) for _ in range(250)] + [rnd(150) for _ in range(3000)]
    reads, offs = csr(parts)
    code = lambda s: int("".join(str("ACGT".index(chr(ch))) for ch in s), 4)
    lut = r.permutation(4 ** p).astype(np.uint32)
    j = int(np.nonzero(lut == 0)[0][0])
    lut[j], lut[code(X)] = lut[code(X)], 0
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P, "hash") as c:
        c.set_order(lut)
        n, d = c.count_reads(reads, offs)
        km, ct = sorted_table(*c.result())
        t = c.timings()
    assert t["second_pass_sub_buckets"] >= 1 and t["overflowed_sub_buckets"] == 0
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


@pytest.mark.parametrize("kind", ["hash", "sort", "hash_redo", "hash_spill", "hash_spill_redo"])
def test_count_partitions_subsets(oracle, kind, monkeypatch):
    """Counting a store in disjoint partition subsets (as the reference's
    phase-2 workers do) gives each subset's k-mers; together the oracle's.
    Every third partition makes every partition a group of its own.
    *_redo starts every group with no output room, so each group overflows
    its output and is counted again; *_spill stages each group from pinned
    host memory while the group before counts."""
    kw = {}
    if kind.endswith("_redo"):
        monkeypatch.setenv("GKC_OUT_ESTIMATE", "1")
    if "spill" in kind:
        kw = dict(spill_host=True, batch_bases=150_000)
    kind = kind.split("_")[0]
    k, p, P = 31, 11, 32
    reads, offs = random_reads(51, 80_000, 6000, 150, 0.005)
    _, _, _, po, stream = oracle.skmgen(reads, offs, k, p, P)
    per = [oracle.count(oracle.extract(stream[int(po[q]):int(po[q + 1])], k), 1, U32) for q in range(P)]
    subsets = [np.arange(0, P, 3), np.arange(1, P, 3), np.arange(2, P, 3)]
    with counter(k, p, P, kind, **kw) as c:
        c.add_reads(reads, offs)
        tot = 0
        for i, sub in enumerate(subsets):
            n, d = c.count_partitions(sub)
            km, ct = sorted_table(*c.result())
            rk, rc = sorted_table(np.concatenate([per[q][0] for q in sub]), np.concatenate([per[q][1] for q in sub]))
            assert d == sum(per[q][2] for q in sub)
            assert np.array_equal(km, rk) and np.array_equal(ct, rc)
            tot += d
            if i == 0:
                with pytest.raises(Exception):
                    c.count_partitions([int(sub[0])])        # counted twice
                with pytest.raises(Exception):
                    c.add_reads(reads, offs)                  # store partly counted
        assert tot == sum(x[2] for x in per)
        assert c.store_stats()[2].sum() == 0                  # released after the last subset


@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_uneven_host_batches(oracle, kind):
    """Host reads of mixed lengths in caller-chosen batches of uneven size give
    the oracle's partitions and counts; every batch reports its latency."""
    k, p, P = 31, 11, 64
    r = np.random.default_rng(71)
    short, so = random_reads(72, 200_000, 20_000, 150, 0.003)
    long_, lo = random_reads(73, 200_000, 60, (1000, 20_000), 0.02)
    reads, offs = csr([short[int(so[i]):int(so[i + 1])].tobytes() for i in range(len(so) - 1)] +
                      [long_[int(lo[i]):int(lo[i + 1])].tobytes() for i in range(len(lo) - 1)])
    perm = r.permutation(len(offs) - 1)
    reads, offs = csr([reads[int(offs[i]):int(offs[i + 1])].tobytes() for i in perm])
    n = len(offs) - 1
    cuts = np.sort(r.choice(np.arange(1, n), 6, replace=False))
    batch_reads = np.diff(np.concatenate([[0], cuts, [n]])).astype(np.uint64)
    pbo, pso, pko, _, _ = oracle.skmgen(reads, offs, k, p, P)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    ko, co = sorted_table(ko, co)
    with counter(k, p, P, kind) as c:
        c.add_reads_batches(reads, offs, batch_reads)
        t = c.batch_timings()
        assert len(t) == len(batch_reads) and (t > 0).all()
        pb, ps, pk = c.store_stats()
        assert np.array_equal(pb, pbo) and np.array_equal(ps, pso) and np.array_equal(pk, pko)
        n_out, d = c.count(2, U32)
        km, ct = sorted_table(*c.result())
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


def test_capacity_overflow_is_redone(oracle):
    """With k = p every position starts a superkmer: far more superkmers and
    bytes per base than phase 1 preallocates, so each batch overflows and is
    redone with exact sizes; results match the oracle."""
    k, p, P = 11, 11, 16
    reads, offs = random_reads(81, 30_000, 3000, 150, 0.01)
    pbo, pso, pko, _, _ = oracle.skmgen(reads, offs, k, p, P)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P)
    ko, co = sorted_table(ko, co)
    import torch
    for device_input in (False, True):  # host batches, then device batches
        with counter(k, p, P, "hash", batch_bases=100_000) as c:
            if device_input:
                c.add_reads(torch.from_numpy(reads).cuda(), torch.from_numpy(offs.view(np.int64)).cuda())
            else:
                c.add_reads(reads, offs)
            pb, ps, pk = c.store_stats()
            assert pso.sum() > offs[-1] // 2  # ~one superkmer per base
            assert np.array_equal(pb, pbo) and np.array_equal(ps, pso) and np.array_equal(pk, pko)
            n_out, d = c.count()
            km, ct = sorted_table(*c.result())
        assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)
