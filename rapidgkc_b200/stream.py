"""Streamed counting at genome scale: reads arrive from the host in batches,
the partition store is spilled to pinned host memory, and phase 2 counts the
partitions in groups staged back to the device.

This is the human-scale configuration: a 3.1 Gbp genome with 50% repeat
content, 30x of 150 bp reads (~93 Gbp), 1 GB batches, learned order.  `scale`
shrinks the genome and the read count together.  Reads are generated batch by
batch from the genome (seeded, as `synth.make_workload` does) by a background
thread, so host memory holds two read batches and the spilled store, never
the whole read set; generation stands in for reading FASTQ from disk and is
reported separately from the counter's time.

    python -m rapidgkc_b200.stream [--scale 0.1] [--batch-gb 1] [--order learned]
"""
from __future__ import annotations

import json
import os
import queue
import threading
import time

import numpy as np

from . import synth
from .capi import KmerCounter


STORE_BYTES_PER_BASE = 1.35  # a spilled chunk keeps its superkmer bytes only


def _mem_available() -> int:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def _device_count_sum(c: KmerCounter, piece: int = 1 << 28) -> int:
    """Sum of the last result's counts, read from device memory in pieces
    through a pinned host buffer (the result can be tens of GB)."""
    import ctypes

    import torch
    kp, cp, n = c.result_device()
    cudart = ctypes.CDLL("libcudart.so.12")  # device pointers are shared through the primary context
    buf = torch.empty(min(n, piece) or 1, dtype=torch.int32, pin_memory=True)
    total = 0
    for i in range(0, n, piece):
        m = min(piece, n - i)
        rc = cudart.cudaMemcpy(ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(cp + 4 * i), ctypes.c_size_t(4 * m),
                               2)  # cudaMemcpyDeviceToHost
        if rc != 0:
            raise RuntimeError(f"cudaMemcpy failed ({rc})")
        total += int(buf[:m].numpy().view(np.uint32).sum(dtype=np.uint64))
    return total


def stream_count(workload: str = "human_3g", scale: float = 1.0, batch_gb: float = 1.0, order: str = "learned",
                 k: int = 31, p: int = 11, partitions: int = 512, cmin: int = 2, spill: bool = True,
                 device: int = 0, threads: int = 0) -> dict:
    w = synth.WORKLOADS[workload]
    spec = synth.GenomeSpec(**{**w["genome"].__dict__})
    spec.length = max(10_000, int(spec.length * scale))
    threads = threads or (os.cpu_count() or 1)
    t0 = time.perf_counter()
    g = synth.genome(spec, w["seed"], threads)
    t_genome = time.perf_counter() - t0
    read_len = 150
    n_reads = max(1, int(w["n_reads"] * scale))
    per_batch = max(1, int(batch_gb * 1e9) // read_len)
    n_batches = (n_reads + per_batch - 1) // per_batch
    q: queue.Queue = queue.Queue(maxsize=1)  # one batch ahead
    gen_s = [0.0]

    def producer():
        for b in range(n_batches):
            nb = min(per_batch, n_reads - b * per_batch)
            t = time.perf_counter()
            item = synth.short_reads(g, nb, read_len, w["err"], w["seed"] + 1 + 7919 * b, pinned=True,
                                     threads=threads)
            gen_s[0] += time.perf_counter() - t
            q.put(item)
        q.put(None)

    # the spilled store takes ~1.3 bytes per base (superkmer bytes; index
    # entries and keys are rebuilt on the device when a range is staged back);
    # it must fit host memory beside two batches
    est_store = int(STORE_BYTES_PER_BASE * n_reads * read_len) if spill else 0
    avail = _mem_available()
    if spill and avail and est_store > 0.8 * avail - 4 * batch_gb * 1e9:
        raise MemoryError(f"a spilled store of ~{est_store / 1e9:.0f} GB does not fit the "
                          f"{avail / 1e9:.0f} GB of available host memory; use a smaller scale")
    th = threading.Thread(target=producer, daemon=True)
    th.start()
    out = {"workload": workload, "scale": scale, "genome_bp": int(spec.length), "reads": n_reads,
           "batches": n_batches, "batch_gb": batch_gb, "order": order, "spill_host": spill, "partitions": partitions}
    with KmerCounter(k=k, p=p, partitions=partitions, counter="hash", spill_host=spill, device=device,
                     batch_bases=int(batch_gb * 1e9) + read_len) as c:
        pin = {"s": 0.0, "bytes": 0, "error": None}
        if spill:
            # pin the store's host memory up front, while the producer makes
            # the first batches: pinning beside the batches competes with
            # them for the driver's lock and the host's cores
            t = time.perf_counter()
            try:
                pin["bytes"] = c.reserve_host(est_store)
            except Exception as e:  # the batches then pin what they need themselves
                pin["error"] = str(e)
            pin["s"] = time.perf_counter() - t
        if order == "learned":
            from .order import default_order_path, load_order
            c.mlp_order(load_order(default_order_path(p))[0])
        bases = 0
        t_add = 0.0
        lat = []
        while True:
            item = q.get()
            if item is None:
                break
            reads, offs = item
            t = time.perf_counter()
            c.add_reads(reads, offs)
            t_add += time.perf_counter() - t
            lat.extend(c.batch_timings().tolist())
            bases += int(offs[-1])
            del reads, offs, item
        th.join()
        pb, ps, pk = c.store_stats()
        c.set_profiling(True)  # per-class kernel times of the count (CUDA events around each launch)
        c.kernel_stats(reset=True)
        t = time.perf_counter()
        kept, distinct = c.count(cmin)
        t_count = time.perf_counter() - t
        tm = c.timings()
        ks = {cls: round(v[0] / 1e3, 4) for cls, v in c.kernel_stats(reset=True).items() if v[1]}
        c.set_profiling(False)
        sum_kept = _device_count_sum(c) if cmin == 2 else None
    out.update({"bases": bases, "store_bytes": int(pb.sum()), "superkmers": int(ps.sum()),
                "kmer_instances": int(pk.sum()), "maxmean_kmers": float(pk.max() / pk.mean()),
                "maxmean_bytes": float(pb.max() / pb.mean()), "kept": kept, "distinct": distinct,
                "phase1_s": t_add, "phase2_s": t_count, "phase2_kernel_s": tm["phase2_kernel_ms"] / 1e3,
                "phase2_stage_s": tm["phase2_stage_ms"] / 1e3, "phase2_groups": tm["phase2_groups"],
                "phase2_kernel_classes_s": ks,
                # threshold >= 2 with no upper bound: every distinct k-mer not
                # kept occurs once, so the kept counts plus the singletons
                # must add up to the k-mer instances
                "instances_check": None if sum_kept is None else {
                    "kept_count_sum": sum_kept, "singletons": distinct - kept,
                    "equal": sum_kept + (distinct - kept) == int(pk.sum())},
                "gbps_incl_pinning": bases / (t_add + t_count + pin["s"]) / 1e9,
                "gbps": bases / (t_add + t_count) / 1e9,
                "batch_latency_ms": {"p50": float(np.percentile(lat, 50)), "max": float(np.max(lat))} if lat else None,
                "generator_s": gen_s[0], "genome_s": t_genome, "host_pinned": pin["bytes"] if spill else 0,
                "pin_s": pin["s"] if spill else 0.0, "pin_error": pin["error"] if spill else None,
                "note": "gbps = bases / (phase 1 calls + count), wall clock; read generation runs beside it on "
                        "another thread; host pinning (pin_s) runs before the first batch"})
    return out


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="streamed, spilled counting of the human-scale workload")
    ap.add_argument("--workload", default="human_3g")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--batch-gb", type=float, default=1.0)
    ap.add_argument("--order", default="learned", choices=["learned", "default"])
    ap.add_argument("--no-spill", action="store_true")
    args = ap.parse_args()
    print(json.dumps(stream_count(args.workload, args.scale, args.batch_gb, args.order, spill=not args.no_spill)),
          flush=True)
