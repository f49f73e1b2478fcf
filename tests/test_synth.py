"""The seeded synthetic workloads that stand in for sequencing data (CPU):
reproducible from the seed, with the composition, read shapes and strand
mix each workload describes."""
import re

import numpy as np

from rapidgkc_b200 import synth

COMP = np.zeros(256, np.uint8)
for a, b in zip(b"ACGT", b"TGCA"):
    COMP[a] = b


def _lowcomp_fraction(g):
    s = g.tobytes()
    pats = [rb"A{50,}", rb"T{50,}", rb"(?:AT){25,}", rb"(?:CAG){17,}", rb"(?:CTG){17,}"]
    return sum(len(m) for p in pats for m in re.findall(p, s)) / len(s)


def test_genome_is_reproducible_and_has_its_gc():
    spec = synth.GenomeSpec(1_000_000, gc=0.41, repeat_frac=0.10, n_families=20)
    a, b = synth.genome(spec, 7), synth.genome(spec, 7)
    assert np.array_equal(a, b) and not np.array_equal(a, synth.genome(spec, 8))
    assert set(np.unique(a).tobytes()) == set(b"ACGT")
    assert abs(np.isin(a, np.frombuffer(b"GC", np.uint8)).mean() - 0.41) < 0.01


def test_low_complexity_runs_follow_the_spec():
    base = dict(length=1_000_000, gc=0.38, repeat_frac=0.15, n_families=20, div_min=0.02, div_max=0.10)
    lc = _lowcomp_fraction(synth.genome(synth.GenomeSpec(**base, lowcomp_frac=0.08), 404))
    none = _lowcomp_fraction(synth.genome(synth.GenomeSpec(**base), 404))
    assert lc > 0.05 and none < 0.005


def test_short_reads_come_from_both_strands():
    g = synth.genome(synth.GenomeSpec(200_000, gc=0.5), 3)
    reads, offs = synth.short_reads(g, 400, 150, 0.0, 11)
    assert np.array_equal(offs, np.arange(401, dtype=np.uint64) * 150)
    fwd = g.tobytes()
    rev = COMP[g[::-1]].tobytes()
    on_fwd = on_rev = 0
    for i in range(400):
        r = reads[150 * i:150 * (i + 1)].tobytes()
        f, v = r in fwd, r in rev
        assert f or v, i  # error-free reads are substrings of one strand
        on_fwd += f
        on_rev += v
    assert 120 < on_fwd < 280 and 120 < on_rev < 280
    # with errors, reads differ from the genome at about the stated rate
    reads_e, _ = synth.short_reads(g, 400, 150, 0.02, 11)
    diff = np.mean(reads_e != reads)
    assert 0.01 < diff < 0.03


def test_long_read_lengths_are_clipped_log_normal():
    lens = synth.long_read_lengths(20_000, 8000.0, 0.5, 1000, 50_000, 5)
    assert lens.min() >= 1000 and lens.max() <= 50_000
    assert abs(np.median(lens) - 8000) < 300


def test_mixed_workload_shape():
    reads, offs = synth.make_workload("mixed_100m", scale=0.005)
    lens = np.diff(offs.astype(np.int64))
    long = lens[lens > 150]
    assert lens.min() == 150 and long.min() >= 1000 and long.max() <= 50_000
    assert abs(long.sum() / lens.sum() - 0.20) < 0.02
    # a bounded sample keeps the genome and draws fewer reads
    r2, o2 = synth.make_workload("bacterial_100m", scale=0.001, read_fraction=0.5)
    r1, o1 = synth.make_workload("bacterial_100m", scale=0.001)
    assert len(o2) - 1 == (len(o1) - 1) // 2 and int(o1[-1]) == 150 * (len(o1) - 1)
