"""The autotuner (rapidgkc_b200/autotune.py): every candidate counts the same
sample and must agree, the fastest is returned and cached, and the options
it picks count the workload exactly like the oracle."""
import numpy as np
import pytest

from conftest import sorted_table

pytestmark = pytest.mark.gpu
U32 = 0xFFFFFFFF


def _sample():
    from rapidgkc_b200 import synth
    return synth.make_workload("mixed_100m", scale=0.002, threads=8)


def test_autotune_picks_a_measured_candidate_and_counts_exactly(oracle):
    from rapidgkc_b200 import KmerCounter
    from rapidgkc_b200.autotune import autotune
    reads, offs = _sample()
    kw = dict(k=31, p=11, cmin=2, partitions=(64, 128), counters=("hash", "sort"), radix_bits=(8, 11),
              orders=("default", "learned"), batch_bases=(1 << 20, 1 << 22), repeats=1)
    res = autotune(reads, offs, **kw)
    o = res["options"]
    # every combination was timed: hash x orders x partitions + sort x digit widths x orders x partitions
    assert len(res["trials"]) == 2 * 2 + 2 * 2 * 2
    assert len(res["batch_trials"]) == 2
    assert o["partitions"] in (64, 128) and o["counter"] in ("hash", "sort") and o["order"] in ("default", "learned")
    assert o["radix_bits"] in (8, 11) and o["batch_bases"] in (1 << 20, 1 << 22)
    best = max(res["trials"], key=lambda t: t["gbps"])
    assert (best["partitions"], best["counter"], best["order"]) == (o["partitions"], o["counter"], o["order"])
    assert autotune(reads, offs, **kw) is res  # cached per sample
    # the chosen options count the sample like the oracle
    ko, co, do, _ = oracle.count_reads(reads, offs, 31, 11, o["partitions"], 2, U32)
    ko, co = sorted_table(ko, co)
    with KmerCounter(k=31, p=11, partitions=o["partitions"], counter=o["counter"], radix_bits=o["radix_bits"],
                     batch_bases=o["batch_bases"]) as c:
        if o["order"] == "learned":
            from rapidgkc_b200.order import default_order_path, load_order
            c.mlp_order(load_order(default_order_path(11))[0])
        n, d = c.count_reads(reads, offs, 2)
        km, ct = sorted_table(*c.result())
    assert d == do and np.array_equal(km, ko) and np.array_equal(ct, co)


def test_autotune_rejects_candidates_that_disagree(monkeypatch):
    """A candidate whose result differs is an error, not a slower choice."""
    from rapidgkc_b200 import autotune as at
    reads, offs = _sample()
    calls = iter(range(100))
    monkeypatch.setattr(at, "_digest", lambda c: next(calls))
    monkeypatch.setattr(at, "_CACHE", {})
    with pytest.raises(RuntimeError, match="results differ"):
        at.autotune(reads, offs, partitions=(64,), counters=("hash",), orders=("default", "learned"),
                    batch_bases=(1 << 22,), repeats=1)
