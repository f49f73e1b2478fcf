"""The reference's .skm partition files (gkc_add_skm, rapidgkc_b200.skmfile):
the reference's own phase-1 output, written as .skm files, loads with the
reference's partition totals and counts to the oracle's table; a store saved
and loaded again counts the same; malformed or mismatched bytes are refused."""
import numpy as np
import pytest

from conftest import sorted_table
from tests_util import random_reads

pytestmark = pytest.mark.gpu
U32 = 0xFFFFFFFF


def _counter(k, p, P, kind="hash", **kw):
    from rapidgkc_b200 import KmerCounter
    return KmerCounter(k=k, p=p, partitions=P, counter=kind, **kw)


@pytest.mark.parametrize("kind", ["hash", "sort"])
def test_reference_phase1_files_count_exactly(oracle, ref_oracle, kind, tmp_path):
    from rapidgkc_b200.skmfile import load_skm, skm_path
    k, p, P = 31, 11, 64
    reads, offs = random_reads(61, 80_000, 6000, (100, 400), 0.01)
    pb, ps, pk, parts = ref_oracle.phase1(reads, offs, k, p, P)
    folder = str(tmp_path) + "/"          # the reference's tmp_file_folder + id + ".skm"
    for i, data in enumerate(parts):
        if len(data) or i % 2:            # some empty partitions have no file at all
            data.tofile(skm_path(folder, i))
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    ko, co = sorted_table(ko, co)
    with _counter(k, p, P, kind) as c:
        assert load_skm(c, folder) == int(pb.sum())
        b, s, km = c.store_stats()
        assert np.array_equal(b, pb) and np.array_equal(s, ps) and np.array_equal(km, pk)
        n, d = c.count(2, U32)
        got = sorted_table(*c.result())
    assert d == do and np.array_equal(got[0], ko) and np.array_equal(got[1], co)


@pytest.mark.parametrize("kind,spill", [("hash", False), ("sort", False), ("hash", True)])
def test_save_and_load_round_trip(kind, spill, tmp_path):
    """A store built in many batches with the learned order, saved as .skm
    files and loaded by a new counter with the same order, counts the same."""
    import torch
    from rapidgkc_b200.order import default_order_path, load_order
    from rapidgkc_b200.skmfile import load_skm, save_skm
    k, p, P = 31, 11, 128
    reads, offs = random_reads(62, 100_000, 8000, (60, 500), 0.01)
    params = load_order(default_order_path(p))[0]
    with _counter(k, p, P, kind, batch_bases=100_000, spill_host=spill) as c:
        c.mlp_order(params)
        c.add_reads(reads, offs)
        stats = c.store_stats()
        nbytes = save_skm(c, str(tmp_path / "skm"))
        n0, d0 = c.count(2, U32)
        ref = sorted_table(*c.result())
    with _counter(k, p, P, kind, spill_host=spill) as c:
        c.mlp_order(params)
        assert load_skm(c, str(tmp_path / "skm")) == nbytes
        for a, b in zip(c.store_stats(), stats):
            assert np.array_equal(a, b)
        n, d = c.count(2, U32)
        assert (n, d) == (n0, d0)
        got = sorted_table(*c.result())
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    # device-resident bytes
    with _counter(k, p, P, kind) as c:
        c.mlp_order(params)
        parts = [np.fromfile(str(tmp_path / "skm" / f"{i}.skm"), np.uint8) for i in range(P)]
        off = np.zeros(P + 1, np.uint64)
        off[1:] = np.cumsum([len(x) for x in parts])
        c.add_skm(torch.from_numpy(np.concatenate(parts)).cuda(), off)
        assert c.count(2, U32) == (n0, d0)


def test_mismatched_or_malformed_bytes_are_refused(oracle):
    k, p, P = 31, 11, 32
    reads, offs = random_reads(63, 30_000, 2000, 150, 0.01)
    _, _, _, po, stream = oracle.skmgen(reads, offs, k, p, P)
    with _counter(k, p, 64) as c:                       # written for 32 partitions
        off = np.concatenate([po, np.full(32, po[-1], np.uint64)])
        with pytest.raises(Exception, match="another partition"):
            c.add_skm(stream, off)
        assert c.store_stats()[2].sum() == 0            # nothing appended
    with _counter(k, p, P) as c:
        bad = po.copy()
        bad[5] += 1                                     # a partition cut inside a superkmer
        with pytest.raises(Exception):
            c.add_skm(stream, bad)
        with pytest.raises(Exception, match="ends inside"):
            c.add_skm(stream[:-1], np.minimum(po, len(stream) - 1))   # the last superkmer cut short
        c.add_skm(stream, po)                           # and the well-formed bytes still load
        ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P)
        n, d = c.count()
        assert d == do
