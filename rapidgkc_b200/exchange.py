"""Multi-GPU counting with a partition exchange: one process per GPU,
torch.distributed for the collectives (NCCL over NVLink on GPUs; gloo moves
CPU tensors through the same code in tests).

The reference counts on one host: its stores never leave the process
(skmstore.hpp:62-279) and phase 2 takes partitions from a shared queue
(gpu_kmercounting.cu:532-535).  Across GPUs the same split holds, because a
k-mer's partition is a function of its minimizer alone (the order is the same
on every rank): counts are exact when every partition is counted by one rank
from every rank's superkmers.

  1. each rank runs phase 1 on its own reads (its store holds all P
     partitions of its reads);
  2. the per-partition k-mer loads are summed over ranks (all_reduce) and
     cut into contiguous ranges of near-equal load, one per rank
     (`partition_ranges`; a learned order makes the loads even, so the
     ranges are about P / world partitions each);
  3. each rank packs its whole store partition-major (`gkc_store_pack`): the
     range owned by rank r is then one contiguous slice of bytes, index and
     keys, so one all_to_all_single per array moves every slice to its owner
     in a single NCCL call (grouped send/recv over NVSwitch);
  4. each rank appends what it received (one chunk per source rank,
     `gkc_store_append`) and counts its range; kept and distinct k-mers are
     summed over ranks.  Each rank's result holds the k-mers of its
     partitions: the global table, sharded by partition.

Received ranges land in the rank's own memory before counting (no kernel
reads a peer's memory).
"""
from __future__ import annotations

import numpy as np

UINT32_MAX = 0xFFFFFFFF


def partition_ranges(loads, world: int) -> np.ndarray:
    """Bounds b[0..world] (b[0] = 0, b[world] = P): rank r owns partitions
    [b[r], b[r+1]).  Each cut is placed where the cumulative load comes
    closest to r / world of the total; all-zero loads are cut by partition
    count."""
    loads = np.asarray(loads, np.float64).reshape(-1)
    P = len(loads)
    if world < 1:
        raise ValueError("world must be >= 1")
    cum = np.cumsum(loads)
    total = float(cum[-1]) if P else 0.0
    if total <= 0:
        return np.array([P * r // world for r in range(world + 1)], np.int64)
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left"))  # cum[b] >= target
        # a cut before partition b leaves cum[b - 1] below it; after it, cum[b]
        below = cum[b - 1] if b > 0 else 0.0
        if b < P and abs(cum[b] - target) < abs(target - below):
            b += 1
        bounds.append(min(max(b, bounds[-1]), P))
    bounds.append(P)
    return np.asarray(bounds, np.int64)


def _collective_device(group, counter_device=None):
    import torch
    import torch.distributed as dist

    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device() if counter_device is None else counter_device)
    return torch.device("cpu")


def exchange_packed(nbytes, idx, keys, counts, bounds, group=None):
    """Moves each owner its range of a packed store.

    nbytes (uint8), idx (int64), keys (int32): this rank's store packed over
    all P partitions (store_pack's layout); counts: uint64 [3, P] per-partition
    bytes, superkmers, k-mers.  Returns, for each source rank in rank order, the
    packed range [bounds[rank], bounds[rank+1]) it sent here:
    (bytes, idx, keys, counts [3, n]) with n partitions."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    counts = np.asarray(counts, np.uint64).reshape(3, -1)
    dev = _collective_device(group, nbytes.device.index if nbytes.is_cuda else None)
    ranges = [(int(bounds[r]), int(bounds[r + 1])) for r in range(world)]
    send = np.array([[counts[0, a:z].sum(), counts[1, a:z].sum()] for a, z in ranges], np.int64).reshape(world, 2)
    recv_t = torch.empty((world, 2), dtype=torch.int64, device=dev)
    dist.all_to_all_single(recv_t, torch.from_numpy(send).to(dev), group=group)
    recv = recv_t.cpu().numpy()
    # the per-partition counts of this rank's range, from every source
    a_me, z_me = ranges[rank]
    n_me = z_me - a_me
    cnt_send = torch.from_numpy(np.concatenate([counts[:, a:z].reshape(-1) for a, z in ranges])
                                .astype(np.int64)).to(dev)
    cnt_recv = torch.empty(3 * n_me * world, dtype=torch.int64, device=dev)
    dist.all_to_all_single(cnt_recv, cnt_send, [3 * n_me] * world, [3 * (z - a) for a, z in ranges], group=group)
    cnt = cnt_recv.cpu().numpy().astype(np.uint64).reshape(world, 3, n_me)
    # the data: one call per array, every source's slice in rank order
    outs = []
    for t, col in ((nbytes, 0), (idx, 1), (keys, 1)):
        t = t if t.device == dev else t.to(dev)
        r = torch.empty(int(recv[:, col].sum()), dtype=t.dtype, device=dev)
        dist.all_to_all_single(r, t, [int(x) for x in recv[:, col]], [int(x) for x in send[:, col]], group=group)
        outs.append(r)
    segs, ob, os_ = [], 0, 0
    for s in range(world):
        nb, ns = int(recv[s, 0]), int(recv[s, 1])
        segs.append((outs[0][ob:ob + nb], outs[1][os_:os_ + ns], outs[2][os_:os_ + ns], cnt[s]))
        ob += nb
        os_ += ns
    return segs


def count_exchanged(counter, cmin: int = 2, cmax: int = UINT32_MAX, group=None) -> dict:
    """Phase 2 across ranks, after every rank's phase 1 (counter.add_reads):
    balances the partitions over the ranks by their global k-mer load,
    exchanges the stores and counts this rank's range.  The counter's result
    then holds the k-mers of this rank's partitions.  Returns
    {"range": (p0, p1), "kept", "distinct" (both summed over ranks),
     "local_kept", "local_distinct", "sent_bytes", "received_bytes"}."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    _, _, pk = counter.store_stats()
    dev = _collective_device(group, counter.device)
    loads = torch.from_numpy(pk.astype(np.int64)).to(dev)
    dist.all_reduce(loads, group=group)
    bounds = partition_ranges(loads.cpu().numpy(), dist.get_world_size(group))
    b, i, k, counts = counter.store_pack()
    counter.store_clear()
    sent = int(b.numel() + 12 * i.numel())
    segs = exchange_packed(b, i, k, counts, bounds, group)
    del b, i, k
    p0, p1 = int(bounds[rank]), int(bounds[rank + 1])
    recv = 0
    for sb, si, sk, sc in segs:
        recv += int(sb.numel() + 12 * si.numel())
        counter.store_append(p0, p1, sb, si, sk, sc)
    del segs
    kept, distinct = counter.count(cmin, cmax)
    tot = torch.tensor([kept, distinct], dtype=torch.int64, device=dev)
    dist.all_reduce(tot, group=group)
    return {"range": (p0, p1), "kept": int(tot[0]), "distinct": int(tot[1]), "local_kept": kept,
            "local_distinct": distinct, "sent_bytes": sent, "received_bytes": recv}
