"""The partition exchange on one GPU: store pack / append between two
counters (two ranks' stores in one process, no collective), and the whole
count_exchanged path with ranks as processes on the same GPU (gloo moves the
packed ranges through host memory; NCCL with one rank).  No kernel waits on
another process."""
import numpy as np
import pytest
import torch.multiprocessing as mp

import dist_workers
from conftest import sorted_table
from tests_util import random_reads

pytestmark = pytest.mark.gpu
U32 = 0xFFFFFFFF


@pytest.mark.parametrize("kind,spill", [("hash", False), ("sort", False), ("hash", True)])
def test_pack_append_between_counters(oracle, kind, spill):
    """Rank r's store is packed over all partitions; each owner appends every
    rank's slice of its range (device tensors, and a host copy for one of
    them) and counts it: the two ranges together give the oracle's table.
    Several batches per rank make several chunks per partition."""
    from rapidgkc_b200 import KmerCounter
    k, p, P = 31, 11, 32
    reads, offs = random_reads(41, 80_000, 6000, (80, 250), 0.01)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    ko, co = sorted_table(ko, co)
    n = len(offs) - 1
    shards = [(reads[:int(offs[n // 2])], offs[:n // 2 + 1]),
              (reads[int(offs[n // 2]):], offs[n // 2:] - offs[n // 2])]
    bounds = [0, 13, P]
    kw = dict(k=k, p=p, partitions=P, counter=kind, spill_host=spill, batch_bases=100_000)
    cs = [KmerCounter(**kw), KmerCounter(**kw)]
    try:
        packs = []
        for c, (r, o) in zip(cs, shards):
            c.add_reads(r, o)
            pb, ps, pk = c.store_stats()
            b, i, kk, cnt = c.store_pack()
            assert np.array_equal(cnt[0], pb) and np.array_equal(cnt[1], ps) and np.array_equal(cnt[2], pk)
            # a sub-range packs to the matching slice of the whole
            b2, i2, k2, cnt2 = c.store_pack(5, 9)
            o0, s0 = int(pb[:5].sum()), int(ps[:5].sum())
            assert np.array_equal(b2.cpu().numpy(), b.cpu().numpy()[o0:o0 + b2.numel()])
            assert np.array_equal(i2.cpu().numpy(), i.cpu().numpy()[s0:s0 + i2.numel()])
            assert np.array_equal(k2.cpu().numpy(), kk.cpu().numpy()[s0:s0 + k2.numel()])
            packs.append((b, i, kk, cnt))
            c.store_clear()
        tot_d, tables = 0, []
        for r, c in enumerate(cs):
            p0, p1 = bounds[r], bounds[r + 1]
            for src, (b, i, kk, cnt) in enumerate(packs):
                o0, o1 = int(cnt[0, :p0].sum()), int(cnt[0, :p1].sum())
                s0, s1 = int(cnt[1, :p0].sum()), int(cnt[1, :p1].sum())
                seg = (b[o0:o1], i[s0:s1], kk[s0:s1], cnt[:, p0:p1])
                if src == 1:  # host memory works too
                    seg = tuple(x.cpu().numpy() if hasattr(x, "cpu") else x for x in seg)
                c.store_append(p0, p1, *seg)
            pk = c.store_stats()[2]
            assert pk[:p0].sum() == 0 and pk[p1:].sum() == 0
            n_, d = c.count(2, U32)
            tot_d += d
            tables.append(c.result())
        km, ct = sorted_table(np.concatenate([t[0] for t in tables]), np.concatenate([t[1] for t in tables]))
        assert tot_d == do and np.array_equal(km, ko) and np.array_equal(ct, co)
    finally:
        for c in cs:
            c.close()


def test_pack_rejects_bad_arguments():
    from rapidgkc_b200 import KmerCounter
    with KmerCounter(k=31, p=11, partitions=16) as c:
        with pytest.raises(Exception):
            c.store_pack(3, 2)
        with pytest.raises(Exception):
            c.store_pack(0, 17)
        b, i, k, cnt = c.store_pack()  # an empty store packs to nothing
        assert b.numel() == 0 and i.numel() == 0 and cnt.shape == (3, 16) and cnt.sum() == 0


@pytest.mark.parametrize("backend,world,kind,spill", [("gloo", 2, "hash", False), ("gloo", 3, "sort", False),
                                                      ("gloo", 2, "hash", True), ("nccl", 1, "hash", False)])
def test_count_exchanged_ranks(backend, world, kind, spill):
    mp.spawn(dist_workers.gpu_exchange, args=(world, dist_workers.free_port(), 43, backend, kind, spill),
             nprocs=world, join=True)


def test_append_to_a_partly_counted_store(oracle):
    """Partition groups arrive one at a time (the reference's phase-2 worker
    counts group after group on its device): a group may be appended after
    other groups were counted, but a counted partition takes no more."""
    from rapidgkc_b200 import KmerCounter
    k, p, P = 31, 11, 16
    reads, offs = random_reads(45, 30_000, 3000, (80, 250), 0.01)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 1, U32)
    ko, co = sorted_table(ko, co)
    with KmerCounter(k=k, p=p, partitions=P) as src, KmerCounter(k=k, p=p, partitions=P) as dst:
        src.add_reads(reads, offs)
        tables, tot = [], 0
        for p0, p1 in ((0, 5), (5, 11), (11, 16)):
            b, i, kk, cnt = src.store_pack(p0, p1)
            dst.store_append(p0, p1, b, i, kk, cnt)
            n_, d = dst.count_partitions(list(range(p0, p1)), 1, U32)
            tables.append(dst.result())
            tot += d
            if p0 == 0:
                with pytest.raises(Exception):
                    dst.store_append(p0, p1, b, i, kk, cnt)  # counted already
        km, ct = sorted_table(np.concatenate([t[0] for t in tables]), np.concatenate([t[1] for t in tables]))
        assert tot == do and np.array_equal(km, ko) and np.array_equal(ct, co)
