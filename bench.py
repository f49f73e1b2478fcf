#!/usr/bin/env python
"""k-mer counting throughput (Gbp/s) of the B200 counter, with the reference
CPU path timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step counts every k-mer of one batch of synthetic reads end to end: reads
-> superkmers -> canonical 31-mers -> counts -> threshold >= 2.  The default
workload is the skewed-partition genome: 200 Mbp at GC 38% with 8%
low-complexity sequence (poly-A, (AT)n, (CAG)n runs of 50-2000 bp) and 15%
repeat families, read as 40M x 150 bp reads at 30x (6 Gbp, 0.3%
substitutions), k=31, m=11, 512 partitions, canonical; it is generated here
from a fixed seed (no public dataset is available).  Its 6 GB of reads exceed
L2, so no L2 flush is needed between steps.

Reported (one JSON line on rank 0):
  value      Gbp/s with the reads already in device memory (whole job, all
             ranks), with the learned minimizer order (rapidgkc_b200/orders,
             trained on skewed genomes of other seeds; --order picks another)
  e2e        the same count through the C ABI from pinned host reads to host
             (k-mer, count) arrays, copies inside the timed region (the library
             packs every other host batch to 2-bit codes on the host's threads
             before copying it; h2d bytes are those it copied)
  orders     default (value order), mix (the learned order's pseudo-random
             bulk order with no network levels) and learned: each timed on the
             device and end to end, with max/mean partition load in k-mers
             and bytes, and whether all (k-mer, count) results are identical
  roofline   the dominant kernel class: algorithmic DRAM bytes per launch /
             CUDA-event launch time, against the measured HBM copy bandwidth
  counting_phase  phase 2 of the hash counter against its compulsory bytes,
             and the sort counter's phase 2 on the same store against the
             LSD-sort byte model (passes of the digit width it uses)
  parity_vs_reference  the reference's own CPU path and this counter on the
             CPU-baseline sample: kept / distinct counts and table digests
  cpu_baseline  the reference's own CPU path (oracle/_ref, compiled from its
             sources) on bounded samples of the same workload, all host cores
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
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "k-mer counting Gbp/s at k=31 on 1 B200, learned vs default order, bit-exact"
WORKLOAD_DESC = {
    "bacterial_100m": "100 Mbp genome GC 41%, 10% repeats (200 families 1-5 kb, 2% div); 20M x 150 bp reads, "
                      "30x, 0.3% subst., both strands",
    "uniform_5m": "5 Mbp uniform genome; 1M x 150 bp reads, 30x, 0.5% subst., both strands",
    "skewed_200m": "200 Mbp genome GC 38%, 8% low-complexity (poly-A, (AT)n, (CAG)n of 50-2000 bp), 15% repeats; "
                   "40M x 150 bp reads, 30x, 0.3% subst., both strands",
    "mixed_100m": "100 Mbp genome; 80% bases from 150 bp reads (0.3%), 20% log-normal long reads (5%)",
}

# DRAM bytes (read + write) per read base of a kernel class, from one ncu
# capture of the current kernels on a 0.05-scale case of the named workload
# (profiles/phase1_and_counter_skewed_small.md, learned order, 256 MiB
# batches): find_superkmers from a full 256 MiB batch (686 MB / 268.4M bases),
# hash_insert (bucket_count_kernel) from its one launch over the whole case
# (846 MB / 300M bases).  The roofline's `traffic` scales them to the bases of
# one launch.  Keyed by (workload, order, kernel class).
TRAFFIC_PER_BASE: dict = {
    ("skewed_200m", "learned", "find_superkmers"): (301.380352e6 + 384.318208e6) / 268435456,
    ("skewed_200m", "learned", "hash_insert"): (739.846144e6 + 105.991424e6) / 300e6,
}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region
    (written to a temporary file, summarised, then removed)."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix=f"gkc_clocks{index}_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
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
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        mx = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def cpu_sample(args, fraction, threads):
    """A bounded sample of the workload: the same genome, `fraction` of its reads."""
    from rapidgkc_b200 import synth
    return synth.make_workload(args.workload, read_fraction=fraction, threads=threads)


def cpu_time(args, reads, offs, threads):
    """The reference's CPU path (oracle/_ref) timed on one sample."""
    from oracle.oracle import RefOracle
    ref = RefOracle(wide=args.k > 32)  # the reference's 128-bit LONGERKMER build for k > 32
    t0 = time.perf_counter()
    d, t1, t2 = ref.run(reads, offs, args.k, args.p, args.partitions, threads)
    wall = time.perf_counter() - t0
    bases = int(offs[-1])
    return {"value": bases / wall / 1e9, "wall_s": wall, "phase1_s": t1, "phase2_s": t2, "distinct": d,
            "bases": bases, "reads": len(offs) - 1}


def cpu_baseline(args, threads, samples):
    """The reference's CPU path on bounded samples of the workload (the last
    one is the reported value; the others show how flat it is in size)."""
    runs = {f: cpu_time(args, r, o, threads) for f, (r, o) in samples.items()}
    fmax = max(runs)
    b = runs[fmax]
    return {"value": b["value"], "unit": "Gbp/s", "cores": threads, "kind": "reference",
            "sample": f"{b['reads']} reads ({b['bases'] / 1e6:.0f} Mbp, {fmax:.0%} of the workload's reads, same "
                      f"genome); reference cpu_funcs.cpp phase 1 + KmerCountingCPU per partition, in-tree MSD radix "
                      f"sort (RADULS not in the reference build); wall {b['wall_s']:.1f} s (phase1 "
                      f"{b['phase1_s']:.1f} s, phase2 {b['phase2_s']:.1f} s); {b['distinct']} distinct",
            "by_sample_size": {f"{f:g}": {"gbps": round(r["value"], 4), "bases": r["bases"],
                                          "wall_s": round(r["wall_s"], 2)} for f, r in sorted(runs.items())}}


def table_digest(km, ct):
    """Order-independent digest of a (k-mer, count) table: kept, xor, sum of
    k-mer * count (mod 2^64), sum of counts.  A 128-bit k-mer (low, high)
    enters as low ^ high * 0x9E3779B97F4A7C15 (the reference digest's fold)."""
    if km.ndim == 2:
        km = km[:, 0] ^ (km[:, 1] * np.uint64(0x9E3779B97F4A7C15))
    return {"kept": int(len(km)), "xor": int(np.bitwise_xor.reduce(km)) if len(km) else 0,
            "sum_kc": int(np.sum(km * ct.astype(np.uint64), dtype=np.uint64)),
            "sum_c": int(ct.sum(dtype=np.uint64))}


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


def reference_program(args, threads, reads, offs):
    """The reference's own command-line program (its gkc_main.cpp and
    cpu_funcs.cpp, built into oracle/_ref/rapidgkc_on_b200), run CPU-only as
    `-cpuonly -ngpu 0 -im ... -read <FASTQ>` on a bounded sample, timed by
    the wall time it prints (gkc_main.cpp:433).  It includes the reference's
    FASTQ loading, which the GPU path's e2e figure does not."""
    exe = os.path.join(ROOT, "oracle", "_ref", "rapidgkc_on_b200")
    if not os.path.exists(exe) or args.k > 32:
        return None
    with tempfile.TemporaryDirectory() as d:
        fq = os.path.join(d, "sample.fq")
        write_fastq(fq, reads, offs)
        cmd = [exe, "-cpuonly", "-ngpu", "0", "-im", "-k", str(args.k), "-p", str(args.p), "-skm",
               str(args.partitions), "-t", str(threads), "-t2", str(threads), "-tsort", "1", "-read", fq]
        p = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=900)
    if p.returncode != 0:
        return {"unavailable": f"exit {p.returncode}"}
    wall = float(p.stdout.strip().split("\n")[-1])
    m = [l for l in (p.stdout + p.stderr).split("\n") if "Total number of distinct kmers:" in l]
    bases = int(offs[-1])
    return {"value": bases / wall / 1e9, "unit": "Gbp/s", "cores": threads, "wall_s": wall,
            "distinct": int(m[-1].split(":")[-1]) if m else None,
            "sample": f"{len(offs) - 1} reads ({bases / 1e6:.0f} Mbp) as FASTQ",
            "cmd": "rapidgkc_on_b200 -cpuonly -ngpu 0 -im -k K -p P -skm SKM -t T -t2 T -tsort 1 -read sample.fq"}


def run_reference(args, rank, world):
    """The reference arm: the reference's CPU path (oracle/_ref) on a bounded
    sample of the workload per step, all host threads, rank 0 only."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    reads, offs = cpu_sample(args, args.cpu_fraction, threads)
    vals, last = [], None
    for i in range(args.warmup + args.steps):
        b = cpu_time(args, reads, offs, threads)
        if i >= args.warmup:
            vals.append(b["value"])
            last = b
    v = statistics.mean(vals)
    base = {"value": v, "unit": "Gbp/s", "cores": threads, "kind": "reference",
            "sample": f"{last['reads']} reads ({last['bases'] / 1e6:.0f} Mbp, {args.cpu_fraction:.0%} of the "
                      f"workload's reads, same genome) per step; reference cpu_funcs.cpp phase 1 + KmerCountingCPU "
                      f"per partition; {last['distinct']} distinct"}
    small = cpu_sample(args, args.cpu_fraction_small, threads)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Gbp/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u128" if args.k > 32 else "u64", "data": "synthetic",
            "config": {"workload": args.workload, "k": args.k, "p": args.p, "partitions": args.partitions,
                       "threshold": f">={args.cmin}", "sample_fraction": args.cpu_fraction},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "Gbp/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "program": reference_program(args, threads, *small)}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="skewed_200m")
    ap.add_argument("--counter", default="hash", choices=["hash", "sort"])
    ap.add_argument("--k", type=int, default=31)
    ap.add_argument("--p", type=int, default=11)
    ap.add_argument("--partitions", type=int, default=512)
    ap.add_argument("--cmin", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-fraction", type=float, default=0.25,
                    help="fraction of the workload's reads in the CPU baseline's timed sample")
    ap.add_argument("--cpu-fraction-small", type=float, default=0.03,
                    help="a smaller sample, timed too (flatness) and used for the parity check")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-sort-leg", action="store_true", help="skip the sort counter's counting-phase run")
    ap.add_argument("--no-exchange", action="store_true",
                    help="with N > 1, count each rank's reads alone (no partition exchange)")
    ap.add_argument("--order", default="learned", choices=["learned", "mix", "default"],
                    help="minimizer order of the reported value (the others are measured beside it)")
    ap.add_argument("--orders", default="default,mix,learned", help="orders measured")
    ap.add_argument("--radix-bits", type=int, default=0, help="sort counter digit width (0: the library's)")
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
    radix_bits = args.radix_bits
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

    # ---- the orders: rank tables installed before each order's runs ----
    from rapidgkc_b200.order import ORDER_MAX_P, default_order_path, load_order, mix_table
    names = [n for n in args.orders.split(",") if n]
    if args.order not in names:
        names.append(args.order)
    luts = {"default": None}
    if args.p <= ORDER_MAX_P:
        luts["mix"] = mix_table(args.p)
        path = default_order_path(args.p)
        if os.path.exists(path):
            luts["learned"] = c.mlp_order(load_order(path)[0])
    names = [n for n in names if n in luts]
    if args.order not in luts:
        args.order = "default"

    def set_order(name):
        c.set_order(luts[name])

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
        dg = table_digest(*c.result())
        d = [dg["xor"], dg["sum_kc"], dg["sum_c"]]
        if world > 1:
            t = torch.tensor([x - (1 << 64) if x >= 1 << 63 else x for x in d], dtype=torch.int64, device="cuda")
            g = [torch.empty_like(t) for _ in range(world)]
            dist.all_gather(g, t)
            a = np.stack([x.cpu().numpy() for x in g]).view(np.uint64)
            d = [int(np.bitwise_xor.reduce(a[:, 0])), int(np.sum(a[:, 1], dtype=np.uint64)),
                 int(np.sum(a[:, 2], dtype=np.uint64))]
        return d

    def timed(fn, steps):
        """Mean device time (ms) of `steps` calls of fn, CUDA events on the
        counter's stream, max over ranks."""
        torch.cuda.synchronize()
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        res = None
        for _ in range(steps):
            res = fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1) / steps
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, res

    def timed_steps(name):
        set_order(name)
        c.store_clear()
        c.add_reads(d_reads, d_offs)
        pb, ps, pk = c.store_stats()
        c.store_clear()
        for _ in range(args.warmup):
            step_device()
        l0 = c.kernel_launches()
        ms, (n_out, n_dist) = timed(step_device, args.steps)
        return {"gbps": bases * world / (ms / 1e3) / 1e9, "ms_per_step": ms,
                "maxmean_kmers": float(pk.max() / pk.mean()), "maxmean_bytes": float(pb.max() / pb.mean()),
                "superkmers": int(ps.sum()), "store_bytes": int(pb.sum()), "kmer_instances": int(pk.sum()),
                "kept": n_out, "distinct": n_dist,
                "launches": (c.kernel_launches() - l0) // args.steps, "timings": c.timings(),
                "checksum": checksum()}

    # ---- device-resident throughput of every order ----
    with ClockSampler(local) as clk:
        runs = {nm: timed_steps(nm) for nm in names}
    main_run = runs[args.order]
    ms, launches, tstats = main_run["ms_per_step"], main_run["launches"], main_run["timings"]
    n_out, n_dist = main_run["kept"], main_run["distinct"]
    value = main_run["gbps"]
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

    # ---- end to end through the C ABI with host buffers, every order ----
    e2e_by_order = {}
    batching = None
    kw = 2 if args.k > 32 else 1  # u64 words per k-mer
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
        hk = torch.empty((cap, kw) if kw == 2 else cap, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
        hc = torch.empty(cap, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        lats = []

        def step_batched():
            c.store_clear()
            c.add_reads_batches(reads, offs, batch_reads)
            lats.extend(c.batch_timings().tolist())
            if exchange:
                from rapidgkc_b200.exchange import count_exchanged
                no = count_exchanged(c, args.cmin)["kept"]
            else:
                no, _ = c.count(args.cmin)
            c.result_into(hk, hc)
            return no

        for nm in names:
            set_order(nm)
            for _ in range(max(1, args.warmup // 2)):
                step_batched()
            lats.clear()
            ems, no = timed(step_batched, args.steps)
            e2e_by_order[nm] = {"value": bases * world / (ems / 1e3) / 1e9, "unit": "Gbp/s",
                                "h2d_bytes_per_step": c.timings()["h2d_bytes"],
                                "d2h_bytes_per_step": int((8 * kw + 4) * (xinfo.get("local_kept", no)
                                                                          if exchange else no)),
                                "ms_per_step": ems, "path": "gkc_add_reads_batches + gkc_count + gkc_result"}
            if nm == args.order:
                sizes = np.diff(offs[np.concatenate([[0], cuts])].astype(np.int64)) / (1 << 20)
                batching = {"batches_per_step": len(batch_reads), "batch_mb_min": float(sizes.min()),
                            "batch_mb_max": float(sizes.max()),
                            "latency_ms": {"p50": float(np.percentile(lats, 50)),
                                           "p95": float(np.percentile(lats, 95)), "max": float(np.max(lats))},
                            "note": "latency = one batch's host-to-device copy start to its phase-1 end "
                                    "(CUDA events)"}
    elif not args.no_e2e:
        cap = int(n_out * 1.05) + 1024
        hk = torch.empty((cap, kw) if kw == 2 else cap, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
        hc = torch.empty(cap, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)

        def step_host():
            if exchange:
                no, _ = exchanged(reads, offs)
                c.result_into(hk, hc)
                return no
            return c.count_reads(reads, offs, args.cmin, out_kmers=hk, out_counts=hc)[0]

        for nm in names:
            set_order(nm)
            for _ in range(max(1, args.warmup // 2)):
                step_host()
            ems, no = timed(step_host, args.steps)
            e2e_by_order[nm] = {"value": bases * world / (ems / 1e3) / 1e9, "unit": "Gbp/s",
                                "h2d_bytes_per_step": c.timings()["h2d_bytes"],
                                "d2h_bytes_per_step": int((8 * kw + 4) * (xinfo.get("local_kept", no)
                                                                          if exchange else no)),
                                "ms_per_step": ems,
                                "path": "gkc_count_reads (host reads, host result arrays; every other host "
                                        "batch packed to 2-bit codes on the host's threads before its copy)"}
    e2e = e2e_by_order.get(args.order)

    orders = {nm: {k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()
                   if k not in ("timings", "checksum", "launches")} for nm, r in runs.items()}
    for nm in names:
        if nm in e2e_by_order:
            orders[nm]["e2e_gbps"] = round(e2e_by_order[nm]["value"], 4)
            orders[nm]["e2e_ms_per_step"] = round(e2e_by_order[nm]["ms_per_step"], 3)
        orders[nm]["overflowed_sub_buckets"] = runs[nm]["timings"]["overflowed_sub_buckets"]
        orders[nm]["phase1_ms"] = round(runs[nm]["timings"]["phase1_ms"], 2)
        orders[nm]["phase2_ms"] = round(runs[nm]["timings"]["phase2_ms"], 2)
    sums = [runs[nm]["checksum"] for nm in names]
    orders["bit_exact"] = all(s == sums[0] for s in sums)
    if "default" in runs and "learned" in runs:
        orders["speedup_learned_vs_default"] = runs["learned"]["gbps"] / runs["default"]["gbps"]
        if "default" in e2e_by_order and "learned" in e2e_by_order:
            orders["e2e_speedup_learned_vs_default"] = (e2e_by_order["learned"]["value"] /
                                                        e2e_by_order["default"]["value"])
    if "mix" in runs and "learned" in runs:
        orders["speedup_learned_vs_mix"] = runs["learned"]["gbps"] / runs["mix"]["gbps"]

    # the hash counter's context is done: its pooled device memory goes back
    # before the sort counter runs, so the sort's partition groups are sized
    # as in a count of its own
    c.close()
    torch.cuda.empty_cache()

    # ---- counting phase against byte models ----
    hbm, src = peaks()
    N, S = main_run["kmer_instances"], main_run["store_bytes"]
    kbytes = 16 if args.k > 32 else 8
    p2 = tstats["phase2_ms"] / 1e3
    comp = S + (kbytes + 4) * n_out
    counting = {"counter": args.counter, "ms_per_step": tstats["phase2_ms"], "kmer_instances": N,
                "store_bytes": S, "kept": n_out,
                "compulsory_bytes": comp, "compulsory_gbs": comp / p2 / 1e9, "compulsory_frac": comp / p2 / 1e9 / hbm,
                "kmer_instances_per_s": N / p2, "peak_gbs": hbm,
                "note": "compulsory = superkmer bytes read once + a key and a u32 count per kept k-mer; the hash "
                        "counter counts each sub-bucket in shared memory, so it is bound by instruction issue "
                        "(decode, shared-memory probes and atomics), not by DRAM: the per-kernel issue and DRAM "
                        "figures are in profiles/"}
    if args.counter == "hash" and not args.no_sort_leg and world == 1:
        # the sort counter on the same reads and order: its phase 2 against
        # the LSD model (superkmers + key write + a key read and write per
        # digit pass over 2k bits + run-length read + output), digit width
        # as used
        with KmerCounter(k=args.k, p=args.p, partitions=args.partitions, counter="sort", device=local,
                         radix_bits=radix_bits, batch_bases=batch_bases) as cs:
            cs.set_stream(stream)
            cs.set_order(luts[args.order])
            sort_steps = max(1, min(3, args.steps))
            for _ in range(1):
                cs.count_reads(d_reads, d_offs, args.cmin)
            sms_, (s_out, s_dist) = timed(lambda: cs.count_reads(d_reads, d_offs, args.cmin), sort_steps)
            ts = cs.timings()
            s_sum = table_digest(*cs.result())
            cs.set_profiling(True)
            cs.kernel_stats(reset=True)
            cs.count_reads(d_reads, d_offs, args.cmin)
            torch.cuda.synchronize()
            sk = cs.kernel_stats(reset=True)
            rb = cs.radix_bits
        passes = -(-2 * args.k // rb)
        sp2 = ts["phase2_ms"] / 1e3
        model = S + kbytes * N + 2 * kbytes * N * passes + kbytes * N + (kbytes + 4) * s_out
        counting["sort_counter"] = {
            "gbps": bases / (sms_ / 1e3) / 1e9, "ms_per_step": sms_, "phase2_ms": ts["phase2_ms"],
            "radix_bits": rb, "passes": passes, "model_bytes": model, "model_gbs": model / sp2 / 1e9,
            "model_frac": model / sp2 / 1e9 / hbm,
            "classes": {k: {"ms": round(v[0], 3), "launches": v[1],
                            "gbs": round(v[2] / (v[0] / 1e3) / 1e9, 1) if v[0] else 0.0}
                        for k, v in sk.items() if v[1]},
            "checksum_equal": [s_sum["xor"], s_sum["sum_kc"], s_sum["sum_c"]] == main_run["checksum"]}
    dom = max(kstats, key=lambda k: kstats[k][0])
    kms, kl, kb = kstats[dom]
    per_launch_s = kms / 1e3 / max(kl, 1)
    achieved = kb / max(kl, 1) / per_launch_s / 1e9 if kl else 0.0
    classes = {k: {"ms_per_step": v[0] / args.steps, "launches_per_step": v[1] // args.steps,
                   "gbs": (v[2] / (v[0] / 1e3) / 1e9) if v[0] else 0.0}
               for k, v in kstats.items() if v[1]}
    tpb = TRAFFIC_PER_BASE.get((args.workload, args.order, dom))
    launch_bases = bases / max(1, kl // args.steps)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": src,
                "traffic": tpb * launch_bases if tpb else None,
                "traffic_source": ("ncu dram__bytes_read+write per base of the same kernel "
                                   "(profiles/phase1_and_counter_skewed_small.md), scaled to the launch's bases")
                if tpb else "no ncu capture of this kernel on this workload and order",
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
        threads_all = os.cpu_count() or 1
        try:
            samples = {f: cpu_sample(args, f, threads_all) for f in (args.cpu_fraction_small, args.cpu_fraction)}
            # parity on the small sample: the reference's CPU path and this
            # counter (reported counter and order, then the other counter)
            from oracle.oracle import RefOracle
            sr, so = samples[args.cpu_fraction_small]
            ref = RefOracle(wide=args.k > 32).digest(sr, so, args.k, args.p, args.partitions, threads_all,
                                                     args.cmin, 0xFFFFFFFF)
            par = {"sample_reads": len(so) - 1, "sample_bases": int(so[-1]), "reference": ref}
            for cn in ("hash", "sort"):
                with KmerCounter(k=args.k, p=args.p, partitions=args.partitions, counter=cn, device=local,
                                 radix_bits=radix_bits, batch_bases=batch_bases) as cp:
                    cp.set_order(luts[args.order])
                    no, nd = cp.count_reads(sr, so, args.cmin)
                    g = table_digest(*cp.result())
                par[cn] = {"kept_equal": no == ref["kept"] and g["kept"] == ref["kept"],
                           "distinct_equal": nd == ref["distinct"],
                           "checksum_equal": (g["xor"], g["sum_kc"], g["sum_c"]) ==
                                             (ref["xor"], ref["sum_kc"], ref["sum_c"])}
            par["order"] = args.order
            line["parity_vs_reference"] = par
            line["cpu_baseline"] = cpu_baseline(args, threads_all, samples)
        except Exception as ex:  # the reference library is test infrastructure; report why it is absent
            line["cpu_baseline"] = {"value": None, "unavailable": f"{type(ex).__name__}: {ex}"}
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
