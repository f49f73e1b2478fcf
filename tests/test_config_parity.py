"""Parity at the benchmarked workload shapes.

Each benchmarked workload (rapidgkc_b200.synth) is generated at a small scale
with its own seed and features: repeat families at set divergence, GC bias,
low-complexity runs of 50-2000 bp, long reads at 5% substitutions.  The CUDA
path (both counters) is compared bit-exact with

* the reference's own CPU path (oracle/_ref: cpu_funcs.cpp phase 1, its
  extraction and sort, the run-length count of KmerCountingCPU) under the
  default order: per-partition superkmer and k-mer counts and the whole
  thresholded (k-mer, count) table;
* the C restatement (oracle/gkc_oracle.c) under the learned order (the
  committed network's rank table) and the mix order (the learned order's
  bulk order with no network levels): per-partition k-mer counts and the
  table.

Integer work: every comparison is exact."""
import functools
import os

import numpy as np
import pytest

from conftest import sorted_table

pytestmark = pytest.mark.gpu
U32 = 0xFFFFFFFF
THREADS = min(16, os.cpu_count() or 1)

# (workload, scale, read_fraction, k): small enough for the CPU checkers,
# large enough to hold the workload's features (families of 1-5 kb, runs of
# up to 2 kb, long reads of up to 50 kb)
CONFIGS = [
    ("uniform_5m", 0.02, 1.0, 31),
    ("bacterial_100m", 0.004, 1.0, 31),
    ("bacterial_100m", 0.004, 1.0, 25),
    ("mixed_100m", 0.004, 1.0, 31),
    ("skewed_200m", 0.003, 1.0, 31),
    ("human_3g", 0.0004, 0.5, 31),
]
IDS = [f"{w}-k{k}" for w, _, _, k in CONFIGS]
P = 512
CMIN = 2


@functools.lru_cache(maxsize=None)
def workload(name, scale, fraction):
    from rapidgkc_b200 import synth
    return synth.make_workload(name, scale=scale, read_fraction=fraction, threads=THREADS)


@functools.lru_cache(maxsize=None)
def order_luts(p):
    """The rank tables of the mix and learned orders (as gkc_mlp_order makes them)."""
    from rapidgkc_b200 import KmerCounter
    from rapidgkc_b200.order import default_order_path, load_order, mix_table
    with KmerCounter(k=31, p=p, partitions=P) as c:
        learned = c.mlp_order(load_order(default_order_path(p))[0])
    return {"mix": mix_table(p), "learned": learned}


def gpu_count(reads, offs, k, kind, lut=None):
    from rapidgkc_b200 import KmerCounter
    with KmerCounter(k=k, p=11, partitions=P, counter=kind) as c:
        c.set_order(lut)
        c.add_reads(reads, offs)
        pb, ps, pk = c.store_stats()
        n, d = c.count(CMIN, U32)
        km, ct = sorted_table(*c.result())
    assert n == len(km)
    return (pb, ps, pk), d, km, ct


def test_workload_features_present():
    """The small-scale cases keep the features they stand for."""
    r, o = workload("mixed_100m", 0.004, 1.0)
    lens = np.diff(o.astype(np.int64))
    assert lens.max() >= 1000 and (lens == 150).mean() > 0.5  # long reads beside 150 bp ones
    r, o = workload("skewed_200m", 0.003, 1.0)
    s = bytes(r[: min(len(r), 30_000_000)])
    assert b"A" * 60 in s or b"T" * 60 in s  # poly-A runs (either strand)
    assert b"CAG" * 15 in s or b"CTG" * 15 in s  # (CAG)n runs (either strand)


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
def test_default_order_matches_reference(cfg, ref_oracle):
    """Default order, both counters: the reference's own CPU path."""
    name, scale, fraction, k = cfg
    reads, offs = workload(name, scale, fraction)
    pb, ps, pk, _ = ref_oracle.phase1(reads, offs, k, 11, P, THREADS)
    rk, rc, rd, _ = ref_oracle.count_reads(reads, offs, k, 11, P, CMIN, U32, threads=THREADS)
    rk, rc = sorted_table(rk, rc)
    for kind in ("hash", "sort"):
        (gb, gs, gk), d, km, ct = gpu_count(reads, offs, k, kind)
        assert np.array_equal(gb, pb) and np.array_equal(gs, ps) and np.array_equal(gk, pk), kind
        assert d == rd, kind
        assert np.array_equal(km, rk) and np.array_equal(ct, rc), kind


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
@pytest.mark.parametrize("order", ["mix", "learned"])
def test_learned_orders_match_oracle(cfg, order, oracle):
    """Mix and learned orders: the C restatement with the same rank table;
    the table also equals the default order's (the order moves k-mers
    between partitions, never changes their counts)."""
    name, scale, fraction, k = cfg
    reads, offs = workload(name, scale, fraction)
    lut = order_luts(11)[order]
    ok, oc, od, opk = oracle.count_reads(reads, offs, k, 11, P, CMIN, U32, lut=lut)
    ok, oc = sorted_table(ok, oc)
    kinds = ("hash", "sort") if order == "learned" else ("hash",)
    for kind in kinds:
        (_, _, gk), d, km, ct = gpu_count(reads, offs, k, kind, lut)
        assert np.array_equal(gk, opk), kind
        assert d == od and np.array_equal(km, ok) and np.array_equal(ct, oc), kind
    _, d0, k0, c0 = gpu_count(reads, offs, k, "hash")
    assert d0 == od and np.array_equal(k0, ok) and np.array_equal(c0, oc)
