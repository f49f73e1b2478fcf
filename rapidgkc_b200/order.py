"""Learned minimizer order.

The reference chooses minimizers by p-mer value with a fixed filter
(minimizer_filter.h:20, gpu_skmgen.cu:243-252).  On genomes with
low-complexity sequence and AT bias that order sends a large share of all
k-mers to a few minimizers.  Here a small network (one-hot p-mer -> 64 ReLU ->
64 ReLU -> 1, FP32, trained by the library's own CUDA kernels) predicts how
heavy a p-mer is as a minimizer.  The order (gkc_mlp_order) ranks the quarter
of all p-mers with the highest scores last, by score, and every other p-mer
in a fixed pseudo-random order (a bijective mix of its value), which removes
the value order's bias towards A-rich p-mers.  Minimizers then come from
p-mers that are rare in the genome, whose sub-buckets hold few distinct
k-mers and rarely overflow the counter's shared-memory tables.  Phase 1 reads a canonical
table, min(rank(v), rank(rc(v))), one L2-resident read per position.

Training data is the counter's own output.  For each training genome, phase 1
runs with the current order, and gkc_minimizer_loads returns the k-mer load of
every minimizer.  The target of a p-mer is

    t(v) = log2(1 + load(v) * 4^p / N)     (N = k-mer instances of the genome)

averaged over the training genomes.  Training is refined over a few
iterations: each iteration runs phase 1 again with the order just learned, and
its loads are combined with the previous targets by maximum.  A p-mer that
becomes heavy once it is preferred is thereby pushed back.  Every order
yields the same (k-mer, count) multiset, because the canonical minimizer is
taken over both strands; only the partition contents change.
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass, field

import numpy as np

from . import synth
from .capi import KmerCounter, load_library

H = 64
ORDERS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "orders")
ORDER_MIX_KEY = 0x5BD1E995  # the tie-break mix of the learned order (gkc_device.cuh)
ORDER_MAX_P = 15  # the learned order's rank levels need 32 - 2p >= 2 bits (order_mlp.cu)


def param_count(p: int) -> int:
    return int(load_library().gkc_mlp_param_count(p))


def init_params(p: int, seed: int) -> np.ndarray:
    """He-normal weights, zero biases; the layout of gkc_mlp_param_count."""
    r = np.random.default_rng(seed)
    W1 = r.normal(0.0, np.sqrt(2.0 / p), (4 * p, H))
    W2 = r.normal(0.0, np.sqrt(2.0 / H), (H, H))
    w3 = r.normal(0.0, np.sqrt(1.0 / H), H)
    out = np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), w3, [0.0]]).astype(np.float32)
    assert len(out) == param_count(p)
    return out


def mix_bits(x: np.ndarray, bits: int, key: int) -> np.ndarray:
    """The bijection of order_lut_kernel (numpy, for mapping ranks back)."""
    mask = np.uint64((1 << bits) - 1) if bits < 32 else np.uint64(0xFFFFFFFF)
    h = np.uint64(bits // 2 if bits > 1 else 1)
    x = (np.asarray(x, np.uint64) ^ np.uint64(key)) & mask
    x = (x * np.uint64(0x9E3779B1)) & mask
    x ^= x >> h
    x = (x * np.uint64(0x85EBCA77)) & mask
    x ^= x >> h
    return x


def loads_by_pmer(keys_load: np.ndarray, lut: np.ndarray | None) -> np.ndarray:
    """Per-p-mer loads from gkc_minimizer_loads output (indexed by key)."""
    if lut is None:
        return keys_load.astype(np.float64)
    mask = np.uint32(len(keys_load) - 1)
    return keys_load[(lut & mask).astype(np.int64)].astype(np.float64)


def partition_stats(counter: KmerCounter) -> dict:
    pb, ps, pk = counter.store_stats()
    return {"maxmean_kmers": float(pk.max() / max(pk.mean(), 1e-9)),
            "maxmean_bytes": float(pb.max() / max(pb.mean(), 1e-9)),
            "cv_kmers": float(pk.std() / max(pk.mean(), 1e-9))}


@dataclass
class TrainLog:
    iterations: list = field(default_factory=list)


def mix_table(p: int) -> np.ndarray:
    """The learned order with no heavy p-mers: every p-mer at level 0, ranked
    by the tie-break mix alone."""
    return mix_bits(np.arange(4 ** p), 2 * p, ORDER_MIX_KEY).astype(np.uint32)


def train_order(workload: str = "skewed_200m", seeds=range(1, 9), scale: float = 0.05, iterations: int = 3,
                k: int = 31, p: int = 11, partitions: int = 512, epochs: int = 4, batch: int = 8192,
                lr: float = 2e-3, device: int = 0, init_seed: int = 0, threads: int = 0, start: str = "mix",
                verbose: bool = False):
    """Trains the order network on the minimizer loads of `workload` genomes
    drawn with `seeds` (the evaluation genome's seed must not be among them).
    The first loads are measured under `start`: "mix" (the learned order's
    own bulk order, the default) or "default" (the value order).  Returns
    (params, log)."""
    import torch

    data = []
    for s in seeds:
        reads, offs = synth.make_workload(workload, scale=scale, seed=int(s) * 1000 + 17, threads=threads)
        data.append((torch.from_numpy(reads).cuda(device), torch.from_numpy(offs.view(np.int64)).cuda(device)))
    params = init_params(p, init_seed)
    log = TrainLog()
    target = None
    lut = mix_table(p) if start == "mix" else None
    with KmerCounter(k=k, p=p, partitions=partitions, device=device) as c:
        for it in range(iterations + 1):
            c.set_order(lut)
            t_sum = np.zeros(4 ** p)
            stats = []
            for d_reads, d_offs in data:
                c.store_clear()
                c.add_reads(d_reads, d_offs)
                stats.append(partition_stats(c))
                load = loads_by_pmer(c.minimizer_loads(), lut)
                n = load.sum()
                t_sum += np.log2(1.0 + load * (4 ** p) / max(n, 1.0))
                c.store_clear()
            t_it = (t_sum / len(data)).astype(np.float32)
            entry = {"iteration": it, "order": "default" if lut is None else ("mix" if it == 0 else "learned"),
                     "maxmean_kmers": float(np.mean([x["maxmean_kmers"] for x in stats])),
                     "maxmean_bytes": float(np.mean([x["maxmean_bytes"] for x in stats]))}
            if it == iterations:
                log.iterations.append(entry)
                break
            target = t_it if target is None else np.maximum(target, t_it)
            t0 = time.perf_counter()
            params, loss = c.mlp_train(params, target, None, epochs=epochs, batch=batch, lr=lr, seed=it)
            entry.update({"train_loss": loss, "train_s": time.perf_counter() - t0})
            lut = c.mlp_order(params)
            log.iterations.append(entry)
            if verbose:
                print(entry, flush=True)
        c.set_order(None)
    return params, log


def save_order(path: str, params: np.ndarray, p: int, meta: dict) -> None:
    """The parameters with their training metadata (.npz), and as raw
    little-endian float32 beside it (.f32, read by gkc_main -order learned)."""
    np.savez(path, params=params.astype(np.float32), p=np.int32(p), meta=np.array(repr(meta)))
    params.astype("<f4").tofile(os.path.splitext(path)[0] + ".f32")


def load_order(path: str):
    z = np.load(path, allow_pickle=False)
    return z["params"].astype(np.float32), int(z["p"])


def default_order_path(p: int = 11) -> str:
    return os.path.join(ORDERS_DIR, f"skewed_m{p}.npz")


def evaluate_orders(params: np.ndarray | None, workload: str = "skewed_200m", scale: float = 1.0,
                    seed: int | None = None, k: int = 31, p: int = 11, partitions: int = 512,
                    counter: str = "hash", repeats: int = 3, device: int = 0, threads: int = 0) -> dict:
    """Default order against the learned one on one genome: partition load,
    device Gbp/s of a whole count (reads resident on the device), and
    whether the (k-mer, count) results are identical."""
    import torch

    reads, offs = synth.make_workload(workload, scale=scale, seed=seed, threads=threads)
    bases = int(offs[-1])
    d_reads = torch.from_numpy(reads).cuda(device)
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda(device)
    out = {"workload": workload, "scale": scale, "bases": bases, "partitions": partitions, "counter": counter}
    digests = {}
    with KmerCounter(k=k, p=p, partitions=partitions, counter=counter, device=device) as c:
        stream = torch.cuda.Stream(device)
        c.set_stream(stream)
        for name in ("default", "learned"):
            c.set_order(None)
            if name == "learned":
                if params is None:
                    continue
                c.mlp_order(params)
            c.store_clear()
            c.add_reads(d_reads, d_offs)
            st = partition_stats(c)
            c.store_clear()
            c.count_reads(d_reads, d_offs, 2)  # warm-up
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(device)
            ev0.record(stream)
            for _ in range(repeats):
                n_out, n_dist = c.count_reads(d_reads, d_offs, 2)
            ev1.record(stream)
            torch.cuda.synchronize(device)
            ms = ev0.elapsed_time(ev1) / repeats
            km, ct = c.result()
            o = np.argsort(km, kind="stable")
            digests[name] = (n_dist, hash(km[o].tobytes()), hash(ct[o].tobytes()))
            t = c.timings()
            out[name] = {**st, "gbps": bases / (ms / 1e3) / 1e9, "ms": ms, "kept": n_out, "distinct": n_dist,
                         "phase1_ms": t["phase1_ms"], "phase2_ms": t["phase2_ms"],
                         "relisted_sub_buckets": t["overflowed_sub_buckets"]}
        c.set_order(None)
    if "learned" in digests:
        out["identical"] = digests["default"] == digests["learned"]
    return out


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="train / evaluate the learned minimizer order")
    ap.add_argument("--train", action="store_true")
    ap.add_argument("--evaluate", action="store_true")
    ap.add_argument("--workload", default="skewed_200m")
    ap.add_argument("--seeds", default="1,2,3,4,5,6,7,8")
    ap.add_argument("--scale", type=float, default=0.05)
    ap.add_argument("--iterations", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--eval-scale", type=float, default=1.0)
    ap.add_argument("--eval-workloads", default="skewed_200m,bacterial_100m")
    ap.add_argument("--out", default=default_order_path(11))
    args = ap.parse_args()
    if args.train:
        seeds = [int(s) for s in args.seeds.split(",")]
        t0 = time.perf_counter()
        params, log = train_order(args.workload, seeds=seeds, scale=args.scale, iterations=args.iterations,
                                  epochs=args.epochs, verbose=True)
        meta = {"workload": args.workload, "seeds": seeds, "scale": args.scale, "iterations": args.iterations,
                "epochs": args.epochs, "log": log.iterations, "seconds": time.perf_counter() - t0}
        os.makedirs(os.path.dirname(args.out), exist_ok=True)
        save_order(args.out, params, 11, meta)
        print(json.dumps({"trained": args.out, **meta}), flush=True)
    if args.evaluate:
        params = load_order(args.out)[0] if os.path.exists(args.out) else None
        for wl in args.eval_workloads.split(","):
            print(json.dumps(evaluate_orders(params, wl, scale=args.eval_scale)), flush=True)
