#!/usr/bin/env python
"""k-mer counting throughput (Gbp/s) of the B200 counter, with the reference
CPU path timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step counts every k-mer of one batch of synthetic reads end to end: reads
-> superkmers -> canonical 31-mers -> counts -> threshold >= 2.  The default
workload is the 100 Mbp bacterial-to-small-eukaryote genome (GC 41%, 10%
repeat families at 2% divergence) read as 20M x 150 bp reads at 30x (3 Gbp,
0.3% substitutions), k=31, m=11, canonical; it is generated here from a fixed
seed (no public dataset is available).  Its 3 GB of reads exceed L2, so no L2
flush is needed between steps.

Reported (one JSON line on rank 0):
  value      Gbp/s with the reads already in device memory (whole job, all ranks),
             with the learned minimizer order (rapidgkc_b200/orders, trained on
             skewed genomes of other seeds; --order default for the value order)
  orders     the same timed steps with the default and the learned order:
             Gbp/s, max/mean partition load, and whether the two (k-mer,
             count) results are identical (order-independent checksums)
  e2e        Gbp/s through the C ABI from pinned host reads to host (k-mer,
             count) arrays, copies inside the timed region
  roofline   the dominant kernel class: algorithmic DRAM bytes per launch /
             CUDA-event launch time, against the measured HBM copy bandwidth
  cpu_baseline  the reference's own CPU path (oracle/_ref, compiled from its
             sources) on a bounded sample of the same workload, all host cores
With --gpus N > 1 (under torchrun) each rank holds its own read set of the
same size drawn from the same genome (weak scaling) and every step counts the
union exactly: phase 1 per rank, then the partition exchange (one NCCL
all_to_all per packed array sends each partition range to its owner) and the
count of each rank's range (rapidgkc_b200/exchange.py); --no-exchange counts
each rank's reads on their own instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "k-mer counting Gbp/s at k=31 on 1 B200, learned vs default order, bit-exact"
WORKLOAD_DESC = {
    "bacterial_100m": "100 Mbp genome GC 41%, 10% repeats (200 families 1-5 kb, 2% div); 20M x 150 bp reads, "
                      "30x, 0.3% subst., both strands",
    "uniform_5m": "5 Mbp uniform genome; 1M x 150 bp reads, 30x, 0.5% subst., both strands",
    "skewed_200m": "200 Mbp genome GC 38%, 8% low-complexity, 15% repeats; 40M x 150 bp reads, 30x, 0.3% subst.",
    "mixed_100m": "100 Mbp genome; 80% bases from 150 bp reads (0.3%), 20% log-normal long reads (5%)",
}


# DRAM bytes per read base of the main kernels, read+write, from one ncu
# capture of a 300 Mbp case (profiles/phase1_and_counter_bacterial_small.md,
# learned order, 256 MiB batches); the roofline's `traffic` scales them to the
# bases of one launch.
TRAFFIC_PER_BASE = {"find_superkmers": 2.61, "scatter_superkmers": 7.85}  # one launch per batch each


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(", ") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        mx = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def cpu_baseline(args, threads):
    """The reference's CPU path (oracle/_ref) on a bounded sample of the workload."""
    from oracle.oracle import RefOracle
    from rapidgkc_b200 import synth
    ref = RefOracle(wide=args.k > 32)  # the reference's 128-bit LONGERKMER build for k > 32
    reads, offs = synth.make_workload(args.workload, read_fraction=args.cpu_fraction, threads=threads)
    t0 = time.perf_counter()
    d, t1, t2 = ref.run(reads, offs, args.k, args.p, args.partitions, threads)
    wall = time.perf_counter() - t0
    bases = int(offs[-1])
    return {"value": bases / wall / 1e9, "unit": "Gbp/s", "cores": threads, "kind": "reference",
            "sample": f"{len(offs) - 1} reads ({bases / 1e6:.0f} Mbp, {args.cpu_fraction:.1%} of the workload's "
                      f"reads, same genome); reference cpu_funcs.cpp phase 1 + KmerCountingCPU per partition, "
                      f"in-tree MSD radix sort (RADULS not in the reference build); wall {wall:.1f} s "
                      f"(phase1 {t1:.1f} s, phase2 {t2:.1f} s); {d} distinct"}


def write_fastq(path, reads, offs):
    """The reads as FASTQ records (@<index>, the bases, +, a quality line)."""
    n = len(offs) - 1
    lens = np.diff(offs.astype(np.int64))
    with open(path, "wb") as f:
        if n and lens.min() == lens.max():  # one read length: records built as rows
            L = int(lens[0])
            ids = np.char.zfill(np.arange(n).astype("S12"), 12).view(np.uint8).reshape(n, 12)
            rec = np.empty((n, 1 + 12 + 1 + L + 3 + L + 1), np.uint8)
            rec[:, 0] = ord("@")
            rec[:, 1:13] = ids
            rec[:, 13] = 10
            rec[:, 14:14 + L] = np.asarray(reads[:n * L]).reshape(n, L)
            rec[:, 14 + L:17 + L] = np.frombuffer(b"\n+\n", np.uint8)
            rec[:, 17 + L:17 + 2 * L] = ord("I")
            rec[:, 17 + 2 * L] = 10
            f.write(rec.tobytes())
        else:
            for i in range(n):
                s = bytes(reads[int(offs[i]):int(offs[i + 1])])
                f.write(b"@%d\n%s\n+\n%s\n" % (i, s, b"I" * len(s)))


def reference_program(args, threads):
    """The reference's own command-line program (its gkc_main.cpp and
    cpu_funcs.cpp, built into oracle/_ref/rapidgkc_on_b200), run CPU-only as
    `-cpuonly -ngpu 0 -im ... -read <FASTQ>` on the same bounded sample, timed
    by the wall time it prints (gkc_main.cpp:433).  It includes the
    reference's FASTQ loading, which the GPU path's e2e figure does not."""
    import tempfile
    from rapidgkc_b200 import synth
    exe = os.path.join(ROOT, "oracle", "_ref", "rapidgkc_on_b200")
    if not os.path.exists(exe) or args.k > 32:
        return None
    reads, offs = synth.make_workload(args.workload, read_fraction=args.cpu_fraction, threads=threads)
    with tempfile.TemporaryDirectory() as d:
        fq = os.path.join(d, "sample.fq")
        write_fastq(fq, reads, offs)
        cmd = [exe, "-cpuonly", "-ngpu", "0", "-im", "-k", str(args.k), "-p", str(args.p), "-skm",
               str(args.partitions), "-t", str(threads), "-t2", str(threads), "-tsort", "1", "-read", fq]
        p = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=900)
    if p.returncode != 0:
        return {"unavailable": f"exit {p.returncode}"}
    wall = float(p.stdout.strip().split("\n")[-1])
    m = [l for l in p.stderr.split("\n") if "Total number of distinct kmers:" in l]
    bases = int(offs[-1])
    return {"value": bases / wall / 1e9, "unit": "Gbp/s", "cores": threads, "wall_s": wall,
            "distinct": int(m[-1].split(":")[-1]) if m else None,
            "sample": f"{len(offs) - 1} reads ({bases / 1e6:.0f} Mbp) as FASTQ",
            "cmd": "rapidgkc_on_b200 -cpuonly -ngpu 0 -im -k K -p P -skm SKM -t T -t2 T -tsort 1 -read sample.fq"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    vals = []
    base = None
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(args, threads)
        if i >= args.warmup:
            vals.append(b["value"])
            base = b
    v = statistics.mean(vals)
    base["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Gbp/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u128" if args.k > 32 else "u64", "data": "synthetic",
            "config": {"workload": args.workload, "k": args.k, "p": args.p, "partitions": args.partitions,
                       "threshold": ">=2", "sample_fraction": args.cpu_fraction},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "Gbp/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "program": reference_program(args, threads)}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bacterial_100m")
    ap.add_argument("--counter", default="hash", choices=["hash", "sort"])
    ap.add_argument("--k", type=int, default=31)
    ap.add_argument("--p", type=int, default=11)
    ap.add_argument("--partitions", type=int, default=512)
    ap.add_argument("--cmin", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-fraction", type=float, default=0.03)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-exchange", action="store_true",
                    help="with N > 1, count each rank's reads alone (no partition exchange)")
    ap.add_argument("--order", default="learned", choices=["learned", "default"],
                    help="minimizer order of the reported value (the other is measured beside it)")
    ap.add_argument("--autotune", default=None, action=argparse.BooleanOptionalAction,
                    help="pick partitions / counter / digit width / order / host batch size on a 10%% sample "
                         "(default: on for mixed_100m)")
    ap.add_argument("--batch-mb", default=None,
                    help="end to end through host batches of random size in [lo,hi] MB, e.g. 64,512 "
                         "(default: 64,512 for mixed_100m)")
    args = ap.parse_args()
    if args.workload == "mixed_100m":
        args.autotune = True if args.autotune is None else args.autotune
        args.batch_mb = "64,512" if args.batch_mb is None else args.batch_mb

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    from rapidgkc_b200 import KmerCounter, synth

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    threads = max(1, (os.cpu_count() or 1) // max(1, world))
    t_gen = time.perf_counter()
    reads, offs = synth.make_workload(args.workload, scale=args.scale, pinned=True, threads=threads,
                                      read_seed=rank)
    t_gen = time.perf_counter() - t_gen
    bases = int(offs[-1])
    tuned = None
    batch_bases = 1 << 28  # 256 MiB phase-1 batches: host copies pipeline finely, scatter slices stay in L2
    radix_bits = 8
    if args.autotune:
        from rapidgkc_b200.autotune import autotune
        n_s = max(1, (len(offs) - 1) // 10)
        s_reads = np.ascontiguousarray(reads[: int(offs[n_s])])
        s_offs = np.ascontiguousarray(offs[: n_s + 1])
        tuned = autotune(s_reads, s_offs, k=args.k, p=args.p, cmin=args.cmin, device=local)
        o = tuned["options"]
        args.partitions, args.counter, args.order = o["partitions"], o["counter"], o["order"]
        batch_bases, radix_bits = o["batch_bases"], o["radix_bits"]
    d_reads = torch.from_numpy(reads).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    stream = torch.cuda.Stream()
    c = KmerCounter(k=args.k, p=args.p, partitions=args.partitions, counter=args.counter, device=local,
                    radix_bits=radix_bits, batch_bases=batch_bases)
    c.set_stream(stream)
    learned_params = None
    if args.order == "learned":
        from rapidgkc_b200.order import default_order_path, load_order
        learned_params = load_order(default_order_path(args.p))[0]

    def set_order(name):
        c.set_order(None)
        if name == "learned":
            c.mlp_order(learned_params)

    exchange = world > 1 and not args.no_exchange
    xinfo = {}

    def exchanged(r, o):
        """Phase 1 of this rank's reads, then the partition exchange and the
        count of this rank's range; (kept, distinct) of the whole job."""
        from rapidgkc_b200.exchange import count_exchanged
        c.store_clear()
        c.add_reads(r, o)
        res = count_exchanged(c, args.cmin)
        xinfo.update(res)
        return res["kept"], res["distinct"]

    def step_device():
        if exchange:
            return exchanged(d_reads, d_offs)
        return c.count_reads(d_reads, d_offs, args.cmin)

    def checksum():
        """Order-independent digest of the (k-mer, count) result (of the
        whole job: every rank holds its partitions' k-mers)."""
        km, ct = c.result()
        if km.ndim == 2:  # k > 32: (low, high) words folded into one u64 per k-mer
            km = km[:, 0] ^ (km[:, 1] * np.uint64(0x9E3779B97F4A7C15))
        d = [int(np.bitwise_xor.reduce(km)) if len(km) else 0,
             int(np.sum(km * ct.astype(np.uint64), dtype=np.uint64)), int(ct.sum(dtype=np.uint64))]
        if world > 1:
            t = torch.tensor([x - (1 << 64) if x >= 1 << 63 else x for x in d], dtype=torch.int64, device="cuda")
            g = [torch.empty_like(t) for _ in range(world)]
            dist.all_gather(g, t)
            a = np.stack([x.cpu().numpy() for x in g]).view(np.uint64)
            d = [int(np.bitwise_xor.reduce(a[:, 0])), int(np.sum(a[:, 1], dtype=np.uint64)),
                 int(np.sum(a[:, 2], dtype=np.uint64))]
        return d

    def timed_steps(name):
        set_order(name)
        c.store_clear()
        c.add_reads(d_reads, d_offs)
        pb, ps, pk = c.store_stats()
        c.store_clear()
        for _ in range(args.warmup):
            step_device()
        torch.cuda.synchronize()
        barrier()
        l0 = c.kernel_launches()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            n_out, n_dist = step_device()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1) / args.steps
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return {"gbps": bases * world / (ms / 1e3) / 1e9, "ms_per_step": ms,
                "maxmean_kmers": float(pk.max() / pk.mean()), "maxmean_bytes": float(pb.max() / pb.mean()),
                "superkmers": int(ps.sum()), "store_bytes": int(pb.sum()), "kmer_instances": int(pk.sum()),
                "kept": n_out, "distinct": n_dist,
                "launches": (c.kernel_launches() - l0) // args.steps, "timings": c.timings(),
                "checksum": checksum()}

    # ---- device-resident throughput, default order, then the learned one ----
    names = ["default"] + (["learned"] if learned_params is not None else [])
    with ClockSampler(local) as clk:
        runs = {nm: timed_steps(nm) for nm in names}
    main_run = runs[args.order]
    ms, launches, tstats = main_run["ms_per_step"], main_run["launches"], main_run["timings"]
    n_out, n_dist = main_run["kept"], main_run["distinct"]
    value = main_run["gbps"]
    orders = {nm: {k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()
                   if k not in ("timings", "checksum", "launches")} for nm, r in runs.items()}
    if len(runs) == 2:
        orders["bit_exact"] = runs["default"]["checksum"] == runs["learned"]["checksum"]
        orders["speedup"] = runs["learned"]["gbps"] / runs["default"]["gbps"]
    # per-kernel-class device times: the same steps again with every launch
    # bracketed by events (kept out of the timed regions above)
    set_order(args.order)
    c.set_profiling(True)
    c.kernel_stats(reset=True)
    for _ in range(args.steps):
        step_device()
    torch.cuda.synchronize()
    kstats = c.kernel_stats(reset=True)
    c.set_profiling(False)

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    batching = None
    if not args.no_e2e and args.batch_mb:
        # host batches of random size in [lo, hi] MB (whole reads), one pipeline
        lo_mb, hi_mb = (float(x) for x in args.batch_mb.split(","))
        rng = np.random.default_rng(11)
        cuts, pos = [], 0
        while pos < bases:
            target = pos + int(rng.uniform(lo_mb, hi_mb) * (1 << 20))
            r1 = int(np.searchsorted(offs, min(target, bases), side="right")) - 1
            r1 = max(r1, (cuts[-1] if cuts else 0) + 1)
            cuts.append(min(r1, len(offs) - 1))
            pos = int(offs[cuts[-1]])
        batch_reads = np.diff(np.concatenate([[0], cuts])).astype(np.uint64)
        cap = int(n_out * 1.05) + 1024
        kw = 2 if args.k > 32 else 1  # u64 words per k-mer
        hk = torch.empty((cap, kw) if kw == 2 else cap, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
        hc = torch.empty(cap, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)

        def step_batched():
            c.store_clear()
            c.add_reads_batches(reads, offs, batch_reads)
            lat = c.batch_timings()
            if exchange:
                from rapidgkc_b200.exchange import count_exchanged
                no = count_exchanged(c, args.cmin)["kept"]
            else:
                no, _ = c.count(args.cmin)
            c.result_into(hk, hc)
            return no, lat

        for _ in range(max(1, args.warmup // 2)):
            step_batched()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        lats = []
        e0.record(stream)
        for _ in range(args.steps):
            no, lat = step_batched()
            lats.extend(lat.tolist())
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / args.steps
        if world > 1:
            t = torch.tensor([ems], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": bases * world / (ems / 1e3) / 1e9, "unit": "Gbp/s",
               "h2d_bytes_per_step": int(len(reads) + 8 * len(offs)),
               "d2h_bytes_per_step": int((8 * kw + 4) * (xinfo.get("local_kept", no) if exchange else no)),
               "ms_per_step": ems, "path": "gkc_add_reads_batches + gkc_count + gkc_result"}
        sizes = np.diff(offs[np.concatenate([[0], cuts])].astype(np.int64)) / (1 << 20)
        batching = {"batches_per_step": len(batch_reads), "batch_mb_min": float(sizes.min()),
                    "batch_mb_max": float(sizes.max()),
                    "latency_ms": {"p50": float(np.percentile(lats, 50)), "p95": float(np.percentile(lats, 95)),
                                   "max": float(np.max(lats))},
                    "note": "latency = one batch's host-to-device copy start to its phase-1 end (CUDA events)"}
    elif not args.no_e2e:
        cap = int(n_out * 1.05) + 1024
        kw = 2 if args.k > 32 else 1  # u64 words per k-mer
        hk = torch.empty((cap, kw) if kw == 2 else cap, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
        hc = torch.empty(cap, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        def step_host():
            if exchange:
                no, _ = exchanged(reads, offs)
                c.result_into(hk, hc)
                return no, None
            return c.count_reads(reads, offs, args.cmin, out_kmers=hk, out_counts=hc)

        for _ in range(max(1, args.warmup // 2)):
            step_host()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            no, _ = step_host()
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / args.steps
        if world > 1:
            t = torch.tensor([ems], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": bases * world / (ems / 1e3) / 1e9, "unit": "Gbp/s",
               "h2d_bytes_per_step": int(len(reads) + 8 * len(offs)),
               "d2h_bytes_per_step": int((8 * kw + 4) * (xinfo.get("local_kept", no) if exchange else no)),
               "ms_per_step": ems}

    # ---- roofline of the dominant kernel class ----
    hbm, src = peaks()
    # counting phase (phase 2) against byte models: the compulsory traffic
    # (superkmer bytes read once + output records of a key and a u32 count)
    # and the LSD-sort path's (superkmers + key write + a key read and write
    # per k-mer per 8-bit digit pass over 2k bits + run-length read + output);
    # keys are 8 B, 16 B for k > 32
    N, S = main_run["kmer_instances"], main_run["store_bytes"]
    p2 = tstats["phase2_ms"] / 1e3
    passes = -(-2 * args.k // 8)
    kbytes = 16 if args.k > 32 else 8
    comp = S + (kbytes + 4) * n_out
    sort_model = S + kbytes * N + 2 * kbytes * N * passes + kbytes * N + (kbytes + 4) * n_out
    counting = {"ms_per_step": tstats["phase2_ms"], "kmer_instances": N, "store_bytes": S,
                "compulsory_bytes": comp, "compulsory_gbs": comp / p2 / 1e9,
                "sort_model_bytes": sort_model, "sort_model_gbs": sort_model / p2 / 1e9,
                "sort_model_frac": sort_model / p2 / 1e9 / hbm, "peak_gbs": hbm}
    dom = max(kstats, key=lambda k: kstats[k][0])
    kms, kl, kb = kstats[dom]
    per_launch_s = kms / 1e3 / max(kl, 1)
    achieved = kb / max(kl, 1) / per_launch_s / 1e9 if kl else 0.0
    classes = {k: {"ms_per_step": v[0] / args.steps, "launches_per_step": v[1] // args.steps,
                   "gbs": (v[2] / (v[0] / 1e3) / 1e9) if v[0] else 0.0}
               for k, v in kstats.items() if v[1]}
    tpb = TRAFFIC_PER_BASE.get(dom) if args.workload == "bacterial_100m" and args.order == "learned" else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": src,
                "traffic": tpb * bases / max(1, kl // args.steps) if tpb else None,
                "traffic_source": "ncu dram__bytes_read+write per base (a 268 Mbp batch of a 300 Mbp case), "
                                  "scaled to the launch's bases" if tpb else None,
                "bytes_per_launch": kb / max(kl, 1), "launch_ms": per_launch_s * 1e3, "classes": classes}

    line = {"metric": METRIC, "value": value, "unit": "Gbp/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u128" if args.k > 32 else "u64", "data": "synthetic",
            "config": {"workload": args.workload, "desc": WORKLOAD_DESC.get(args.workload, ""),
                       "bases_per_rank": bases, "reads_per_rank": len(offs) - 1, "k": args.k, "p": args.p,
                       "partitions": args.partitions, "counter": args.counter, "order": args.order,
                       "batch_bases": batch_bases,
                       "threshold": f">={args.cmin}",
                       "parallelism": f"dp{world} reads + partition exchange" if exchange
                       else f"dp{world} (independent read sets)",
                       "l2": f"inputs ({bases / 1e9:.1f} GB) larger than L2; no flush", "kmers_kept": n_out,
                       "distinct": n_dist, "gen_s": round(t_gen, 1),
                       "sub_buckets": tstats["sub_buckets"], "overflowed": tstats["overflowed_sub_buckets"],
                       "phase1_ms": round(tstats["phase1_ms"], 2), "phase2_ms": round(tstats["phase2_ms"], 2)},
            "orders": orders, "roofline": roofline, "counting_phase": counting, "e2e": e2e,
            "gpu_launches": int(launches)}
    if exchange and xinfo:
        line["exchange"] = {"partitions_rank0": list(xinfo["range"]), "sent_bytes_rank0": xinfo["sent_bytes"],
                            "received_bytes_rank0": xinfo["received_bytes"],
                            "note": "kept/distinct are of the union of all ranks' reads"}
    if batching:
        line["batching"] = batching
    if tuned:
        line["autotune"] = {"options": tuned["options"], "sample_gbps": tuned["gbps"],
                            "trials": len(tuned["trials"]) + len(tuned["batch_trials"])}
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if rank == 0 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(args, os.cpu_count() or 1)
        except Exception as ex:  # the reference library is test infrastructure; report why it is absent
            line["cpu_baseline"] = {"value": None, "unavailable": str(ex)}
    c.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
