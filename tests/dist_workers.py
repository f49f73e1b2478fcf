"""Rank bodies for the multi-process exchange tests (started with
torch.multiprocessing.spawn, one process per rank, rendezvous on 127.0.0.1).
A failed check raises in the rank, and spawn re-raises it in the test."""
import datetime
import os
import socket

import numpy as np

from tests_util import random_reads


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, backend):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))


def _shard(reads, offs, rank, world):
    n = len(offs) - 1
    a, z = n * rank // world, n * (rank + 1) // world
    return reads[int(offs[a]):int(offs[z])].copy(), (offs[a:z + 1] - offs[a]).astype(np.uint64)


def _range_table(o, reads, offs, k, p, P, p0, p1, cmin):
    """The single-process oracle's (k-mers, counts, distinct) of partitions [p0, p1)."""
    _, _, _, po, st = o.skmgen(reads, offs, k, p, P)
    return o.count(o.extract(st[int(po[p0]):int(po[p1])], k), cmin)


def oracle_exchange(rank, world, port, seed, k=25):
    """Each rank packs the oracle's phase-1 output of its read shard (the
    partition streams, with an index tagging the source rank and keys naming
    each superkmer's partition), exchanges it with exchange_packed over gloo,
    and counts its range with the oracle: the result must equal the
    single-process oracle's for that range, and the distinct totals must add
    up to the whole input's.  k > 32 gives 128-bit (low, high) k-mer tables."""
    import torch
    import torch.distributed as dist

    _init(rank, world, port, "gloo")
    try:
        from oracle.oracle import Oracle
        from rapidgkc_b200.exchange import exchange_packed, partition_ranges

        o = Oracle()
        p, P = 9, 24
        reads, offs = random_reads(seed, 20_000, 1500, (40, 200), 0.01)
        sr, so = _shard(reads, offs, rank, world)
        pb, ps, pk, _, stream = o.skmgen(sr, so, k, p, P)
        counts = np.stack([pb, ps, pk])
        part = np.repeat(np.arange(P), ps.astype(np.int64))
        idx = (np.int64(rank) << np.int64(40)) | np.arange(len(part), dtype=np.int64)
        keys = part.astype(np.int32)
        loads = torch.from_numpy(pk.astype(np.int64))
        dist.all_reduce(loads)
        bounds = partition_ranges(loads.numpy(), world)
        segs = exchange_packed(torch.from_numpy(stream), torch.from_numpy(idx), torch.from_numpy(keys), counts,
                               bounds)
        p0, p1 = int(bounds[rank]), int(bounds[rank + 1])
        assert len(segs) == world
        for s, (sb, si, sk, sc) in enumerate(segs):
            assert sc.shape == (3, p1 - p0)
            assert np.array_equal(sk.numpy(), np.repeat(np.arange(p0, p1), sc[1].astype(np.int64)))
            assert np.all((si.numpy() >> 40) == s)
            assert sb.numel() == int(sc[0].sum())
        parts = []
        for j in range(p1 - p0):
            for sb, _, _, sc in segs:
                b0 = int(sc[0, :j].sum())
                parts.append(sb.numpy()[b0:b0 + int(sc[0, j])])
        got = o.count(o.extract(np.concatenate(parts) if parts else np.zeros(0, np.uint8), k), 1)
        exp = _range_table(o, reads, offs, k, p, P, p0, p1, 1)
        assert got[2] == exp[2] and np.array_equal(got[0], exp[0]) and np.array_equal(got[1], exp[1])
        t = torch.tensor([got[2]], dtype=torch.int64)
        dist.all_reduce(t)
        _, _, _, _, st = o.skmgen(reads, offs, k, p, P)
        assert int(t[0]) == o.count(o.extract(st, k), 1)[2]
    finally:
        dist.destroy_process_group()


def gpu_exchange(rank, world, port, seed, backend, kind, spill):
    """The whole multi-rank path on the GPU: phase 1 of the rank's shard,
    count_exchanged (pack, exchange, append, count), against the oracle's
    table of the rank's partition range and its global totals."""
    import torch.distributed as dist

    _init(rank, world, port, backend)
    try:
        import torch

        from oracle.oracle import Oracle
        from rapidgkc_b200 import KmerCounter
        from rapidgkc_b200.exchange import count_exchanged

        torch.cuda.set_device(0)
        o = Oracle()
        k, p, P = 31, 11, 64
        reads, offs = random_reads(seed, 60_000, 5000, (100, 300), 0.01)
        sr, so = _shard(reads, offs, rank, world)
        with KmerCounter(k=k, p=p, partitions=P, counter=kind, spill_host=spill, batch_bases=200_000) as c:
            c.add_reads(sr, so)
            res = count_exchanged(c, cmin=2)
            km, ct = c.result()
        p0, p1 = res["range"]
        ek, ec, ed = _range_table(o, reads, offs, k, p, P, p0, p1, 2)
        order = np.argsort(km, kind="stable")
        assert res["local_distinct"] == ed and res["local_kept"] == len(ek)
        assert np.array_equal(km[order], ek) and np.array_equal(ct[order], ec)
        ko, _, do, _ = o.count_reads(reads, offs, k, p, P, 2)
        assert res["distinct"] == do and res["kept"] == len(ko)
    finally:
        dist.destroy_process_group()
