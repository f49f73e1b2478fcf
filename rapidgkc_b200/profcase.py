"""One small count of a named workload, for profiler captures: the reads are
generated, copied to the device, and counted `reps` times with the chosen
counter and order, and nothing else runs (few launches, so a profiler that
serialises every launch ends quickly).

    python -m rapidgkc_b200.profcase [--workload skewed_200m] [--scale 0.05]
        [--counter hash|sort] [--order learned|mix|default] [--reps 2] [--k 31]

Prints one JSON line: bases, kept and distinct k-mers, the device time of
the last count (CUDA events), free device memory before the counts, and,
with --classes, each kernel class's time, launches and algorithmic bytes over
one more count with every launch bracketed by events.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="skewed_200m")
    ap.add_argument("--scale", type=float, default=0.05)
    ap.add_argument("--counter", default="hash", choices=["hash", "sort"])
    ap.add_argument("--order", default="learned", choices=["learned", "mix", "default"])
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--k", type=int, default=31)
    ap.add_argument("--p", type=int, default=11)
    ap.add_argument("--partitions", type=int, default=512)
    ap.add_argument("--radix-bits", type=int, default=0)
    ap.add_argument("--batch-mb", type=int, default=256)
    ap.add_argument("--classes", action="store_true", help="also time every kernel class (one more count)")
    args = ap.parse_args()

    import torch
    from . import KmerCounter, synth
    from .order import default_order_path, load_order, mix_table

    reads, offs = synth.make_workload(args.workload, scale=args.scale, threads=os.cpu_count() or 1)
    d_reads = torch.from_numpy(reads).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    with KmerCounter(k=args.k, p=args.p, partitions=args.partitions, counter=args.counter,
                     radix_bits=args.radix_bits, batch_bases=args.batch_mb << 20) as c:
        if args.order == "learned":
            c.mlp_order(load_order(default_order_path(args.p))[0])
        elif args.order == "mix":
            c.set_order(mix_table(args.p))
        stream = torch.cuda.Stream()
        c.set_stream(stream)
        ms = 0.0
        for _ in range(args.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            n_out, n_dist = c.count_reads(d_reads, d_offs, 2)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
        free_b, total_b = torch.cuda.mem_get_info()
        line = {"workload": args.workload, "scale": args.scale, "bases": int(offs[-1]),
                "counter": args.counter, "order": args.order, "kept": n_out, "distinct": n_dist,
                "ms_last": ms, "gbps_last": int(offs[-1]) / ms / 1e6, "launches": c.kernel_launches(),
                "free_gb_after": free_b / 1e9, "timings": c.timings()}
        if args.classes:
            c.set_profiling(True)
            c.kernel_stats(reset=True)
            c.count_reads(d_reads, d_offs, 2)
            torch.cuda.synchronize()
            line["classes"] = {k: {"ms": round(v[0], 3), "launches": v[1],
                                   "gbs": round(v[2] / (v[0] / 1e3) / 1e9, 1) if v[0] else 0.0}
                               for k, v in c.kernel_stats(reset=True).items() if v[1]}
            c.set_profiling(False)
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
