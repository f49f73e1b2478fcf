"""gkc_pack_bases: host batches cross PCIe as 2-bit words, 16 bases to a word,
first base highest.  The words must be exactly those that phase 1 stages from
ASCII on the device, with the device's base map (A/C/G/T in either case ->
0..3; N, U and every other byte -> 0, as the reference reads N and U).  These
run on the CPU: the packer is host code."""
import numpy as np
import pytest

from rapidgkc_b200.capi import pack_bases


def ref_pack(b):
    """The device's base map and word layout, restated with numpy."""
    b = np.asarray(b, np.uint8)
    low = b | 0x20
    ok = (low == ord("a")) | (low == ord("c")) | (low == ord("g")) | (low == ord("t"))
    code = (((b >> 1) ^ (b >> 2)) & 3).astype(np.uint32) * ok
    nw = (len(b) + 15) // 16
    slots = np.zeros(nw * 16, np.uint32)
    slots[:len(b)] = code
    shifts = (30 - 2 * np.arange(16)).astype(np.uint32)
    return np.bitwise_or.reduce(slots.reshape(nw, 16) << shifts, axis=1).astype(np.uint32) if nw else \
        np.zeros(0, np.uint32)


def test_every_byte_value_at_every_slot():
    # each byte value at each of the 16 slots of a word, in both the vector
    # body and the scalar tail (lengths 32k and 32k + 17)
    for extra in (0, 17):
        b = np.repeat(np.arange(256, dtype=np.uint8), 16 * 8)
        b = np.concatenate([b, np.frombuffer(b"ACGTNacgtn"[: extra % 11] * 2, np.uint8)[:extra]])
        assert np.array_equal(pack_bases(b), ref_pack(b))
    # the map itself, one byte at a time
    for v in range(256):
        w = pack_bases(bytes([v]))
        c = chr(v).lower()
        assert w[0] >> 30 == ({"a": 0, "c": 1, "g": 2, "t": 3}.get(c, 0) if v < 128 else 0)


@pytest.mark.parametrize("n", [0, 1, 15, 16, 17, 31, 32, 33, 63, 64, 65, 1000, 65537])
def test_ragged_lengths(n):
    r = np.random.default_rng(n)
    b = np.frombuffer(b"ACGTacgtNnUu-X\n", np.uint8)[r.integers(0, 15, n)]
    assert np.array_equal(pack_bases(b), ref_pack(b))


def test_large_batch_on_the_thread_pool():
    # 40 MB: split over the pool's threads (word ranges), AVX2 where present
    r = np.random.default_rng(7)
    b = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, 40_000_003)]
    b[r.integers(0, len(b), 100_000)] = ord("N")
    b[r.integers(0, len(b), 100_000)] = ord("g")
    assert np.array_equal(pack_bases(b), ref_pack(b))
