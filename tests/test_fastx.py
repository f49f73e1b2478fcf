"""The GPU FASTQ / FASTA record scanner (gkc_parse_fastx, gkc_add_fastx)
against the record rules restated in oracle/fastx_oracle.py: exact reads and
offsets on random text (CRLF, blank lines, wrapped FASTA, lines longer than a
16 KiB tile), text fed in pieces with the FASTQ phase carried, and k-mer counts
of the parsed reads against the oracle's."""
import numpy as np
import pytest

from oracle.fastx_oracle import csr, parse_fastx

U32 = 0xFFFFFFFF


def test_oracle_known_answers():
    assert parse_fastx(b"@r1\nACGT\n+\nIIII\n@r2\nGG\r\n+\nII\n") == ([b"ACGT", b"GG"], 0)
    # the reference's phase carry (fileloader.hpp:222): a piece that starts on a read line
    assert parse_fastx(b"ACGT\n+\nIIII\n@r2\n", "fastq", 1) == ([b"ACGT", b""], 1)
    assert parse_fastx(b">a x\nAC\nGT\n\n>b\nTT\n", "fasta") == ([b"ACGT", b"TT"], 0)
    assert parse_fastx(b"CC\nGG\n>b\nTT", "fasta") == ([b"CCGG", b"TT"], 0)
    # single-line FASTA: every second line, as the reference loader reads it
    assert parse_fastx(b">1\nAAC\n>2\nGGT\n", "fasta")[0] == [b"AAC", b"GGT"]


@pytest.mark.parametrize("fmt", ["fastq", "fasta"])
def test_oracle_pinned_to_the_reference_loader(tmp_path, fmt):
    """The reads the reference's own ReadLoader extracts (fileloader.hpp:51-545,
    1 MB buffers, so records cross buffer boundaries) are the oracle's, in
    order.  The loader skips empty reads, which hold no k-mer; the
    comparison leaves them out.  FASTA is single-line here: the loader takes
    every second line, which agrees with the oracle's records only then."""
    from oracle.oracle import ref_load_reads
    if fmt == "fastq":
        text, _ = random_fastq(5, 9000, lens=(0, 400), crlf=0.0)
        path = tmp_path / "reads.fq"
    else:
        r = np.random.default_rng(3)
        acgt = np.frombuffer(b"ACGTN", np.uint8)
        recs = [bytes(acgt[r.integers(0, 5, int(r.integers(1, 600)))]) for _ in range(6000)]
        text = b"".join(b">r%d desc\n%s\n" % (i, x) for i, x in enumerate(recs))
        path = tmp_path / "reads.fa"
    assert len(text) > 1 << 20
    path.write_bytes(text)
    try:
        got = ref_load_reads(str(path), 1)
    except FileNotFoundError as e:
        pytest.skip(str(e))
    assert got == [x for x in parse_fastx(text, fmt)[0] if x]


def random_fastq(seed, n, lens=(0, 400), crlf=0.1, long_every=0):
    r = np.random.default_rng(seed)
    alpha = np.frombuffer(b"ACGTNacgt", np.uint8)
    out, reads = [], []
    for i in range(n):
        L = int(r.integers(lens[0], lens[1] + 1))
        if long_every and i % long_every == 0:
            L = int(r.integers(20_000, 40_000))
        s = bytes(alpha[r.integers(0, len(alpha), L)])
        eol = b"\r\n" if r.random() < crlf else b"\n"
        out.append(b"@read%d extra\n" % i + s + eol + b"+\n" + b"I" * L + b"\n")
        reads.append(s)
    return b"".join(out), reads


def random_fasta(seed, n, lens=(0, 3000)):
    r = np.random.default_rng(seed)
    alpha = np.frombuffer(b"ACGTN", np.uint8)
    out = []
    for i in range(n):
        L = int(r.integers(lens[0], lens[1] + 1))
        s = bytes(alpha[r.integers(0, len(alpha), L)])
        w = int(r.integers(1, 200)) if r.random() < 0.8 else max(L, 1)
        out.append(b">rec%d\n" % i)
        for j in range(0, L, w):
            out.append(s[j:j + w] + (b"\r\n" if r.random() < 0.1 else b"\n"))
        if r.random() < 0.1:
            out.append(b"\n")
    return b"".join(out)


def _gpu_counter(**kw):
    from rapidgkc_b200 import KmerCounter
    return KmerCounter(k=31, p=11, partitions=64, **kw)


def _check(c, text, fmt, state=0):
    rd, of, st = c.parse_fastx(text, fmt, state)
    ereads, est = parse_fastx(text, fmt, state)
    er, eo = csr(ereads)
    assert st == est and np.array_equal(of, eo) and np.array_equal(rd, er)
    return ereads


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_fastq_matches_oracle(seed):
    text, reads = random_fastq(seed, 3000, long_every=700 if seed == 3 else 0)
    with _gpu_counter() as c:
        got = _check(c, text, "fastq")
        assert got == reads
        for s in range(4):  # any start phase
            _check(c, text[: len(text) // 3], "fastq", s)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [4, 5])
def test_fasta_matches_oracle(seed):
    text = random_fasta(seed, 400)
    with _gpu_counter() as c:
        _check(c, text, "fasta")
        _check(c, b"\n\n" + text, "fasta")
        _check(c, text[len(text) // 2:], "fasta")   # starts inside a record


@pytest.mark.gpu
def test_pieces_carry_the_fastq_phase():
    """A file fed in pieces cut after random newlines gives the oracle's reads
    piece by piece, and, without the empty reads at cuts, the whole file's."""
    text, reads = random_fastq(6, 2000)
    r = np.random.default_rng(7)
    nl = np.flatnonzero(np.frombuffer(text, np.uint8) == ord("\n")) + 1
    cuts = [0] + sorted(r.choice(nl[:-1], 25, replace=False).tolist()) + [len(text)]
    with _gpu_counter() as c:
        state, got = 0, []
        for a, b in zip(cuts[:-1], cuts[1:]):
            piece = text[a:b]
            rd, of, st = c.parse_fastx(piece, "fastq", state)
            ereads, est = parse_fastx(piece, "fastq", state)
            assert st == est and np.array_equal(of, csr(ereads)[1]) and np.array_equal(rd, csr(ereads)[0])
            got += ereads
            state = st
        assert [x for x in got if x] == [x for x in reads if x]


@pytest.mark.gpu
def test_edge_cases():
    with _gpu_counter() as c:
        for text, fmt in [(b"", "fastq"), (b"", "fasta"), (b"@only-a-header", "fastq"), (b">h", "fasta"),
                          (b"\n\n\n", "fastq"), (b"ACGT", "fasta"), (b"@h\nAC", "fastq"), (b"\r\n>\r\n", "fasta")]:
            _check(c, text, fmt)
        with pytest.raises(Exception):
            c.parse_fastx(b"@h\nAC\n", "fastq", 4)   # phase out of range


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["fastq", "fasta"])
def test_add_fastx_counts_match_oracle(oracle, fmt):
    """Phase 1 straight from text (host bytes and a device tensor) counts the
    oracle's reads exactly."""
    import torch
    from tests_util import random_reads
    reads, offs = random_reads(8, 50_000, 4000, (30, 600), 0.01)
    seqs = [reads[int(offs[i]):int(offs[i + 1])].tobytes() for i in range(len(offs) - 1)]
    if fmt == "fastq":
        text = b"".join(b"@r\n" + s + b"\n+\n" + b"#" * len(s) + b"\n" for s in seqs)
    else:
        text = b"".join(b">r\n" + b"\n".join(s[j:j + 70] for j in range(0, len(s), 70)) + b"\n" for s in seqs)
    k, p, P = 31, 11, 64
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32)
    order = np.argsort(ko)
    for dev in (False, True):
        with _gpu_counter() as c:
            t = torch.from_numpy(np.frombuffer(text, np.uint8).copy()).cuda() if dev else text
            nr, nb, _ = c.add_fastx(t, fmt)
            assert nr == len(seqs) and nb == len(reads)
            n, d = c.count(2, U32)
            km, ct = c.result()
            o = np.argsort(km)
            assert d == do and np.array_equal(km[o], ko[order]) and np.array_equal(ct[o], co[order])
