"""gkc_count_keys_noalloc: the raw-key hash count with fixed device scratch and
no allocation, for callers that cannot allocate device memory (a caller that
runs its own memory pool, or one where cudaMalloc / cudaFree would stall the
device mid-pipeline).  Checked through the C ABI against numpy's np.unique
and against gkc_count_keys (the allocating entry point), on consecutive calls
that share the one scratch table.  Collected last on purpose; it also passes
alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

U32 = 0xFFFFFFFF
M64 = (1 << 64) - 1


def _noalloc(L, d_keys, n, cmin, cmax, out_k, out_c, cap):
    no, nd = C.c_uint64(0), C.c_uint64(0)
    rc = L.gkc_count_keys_noalloc(C.c_void_p(d_keys.data_ptr()), n, cmin, cmax, C.c_void_p(out_k.data_ptr()),
                                  C.c_void_p(out_c.data_ptr()), cap, C.byref(no), C.byref(nd), None)
    return rc, no.value, nd.value


def _unhash(h):
    """Inverse of the table's key hash (hash64: xor-shift / multiply rounds),
    so that a test can choose the slot a key lands in."""
    h ^= h >> 33
    h = (h * pow(0x81DADEF4BC2DD44D, -1, 1 << 64)) & M64
    h ^= (h >> 27) ^ (h >> 54)
    h = (h * pow(0x7FB5D329728EA185, -1, 1 << 64)) & M64
    h ^= (h >> 31) ^ (h >> 62)
    return h


def test_unhash_inverts_the_table_hash():
    def hash64(z):
        z ^= z >> 31
        z = (z * 0x7FB5D329728EA185) & M64
        z ^= z >> 27
        z = (z * 0x81DADEF4BC2DD44D) & M64
        z ^= z >> 33
        return z
    for x in (0, 1, 12345, M64 - 1, 0x9E3779B97F4A7C15):
        assert hash64(_unhash(x)) == x


@pytest.mark.gpu
def test_noalloc_matches_unique_and_count_keys_on_consecutive_calls():
    import torch
    from rapidgkc_b200 import KmerCounter
    from rapidgkc_b200.capi import GKC_ELIMIT, load_library
    L = load_library()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    cap = 1 << 19
    out_k = torch.empty(cap, dtype=torch.int64, device=dev)
    out_c = torch.empty(cap, dtype=torch.int32, device=dev)
    r = np.random.default_rng(61)
    # two calls in a row: many repeats with threshold >= 2, then mostly distinct keys in [1, 5]
    for n, span, cmin, cmax in [(400_000, 150_000, 2, U32), (1 << 19, 1 << 40, 1, 5)]:
        keys = r.integers(0, span, n, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        keys[keys == np.uint64(M64)] = 1
        d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
        rc, no, nd = _noalloc(L, d_keys, n, cmin, cmax, out_k, out_c, cap)
        assert rc == 0
        km = out_k[:no].cpu().numpy().view(np.uint64)
        ct = out_c[:no].cpu().numpy().view(np.uint32)
        o = np.argsort(km)
        km, ct = km[o], ct[o]
        # independent reference: numpy's sort-based unique counts
        uk, uc = np.unique(keys, return_counts=True)
        keep = (uc >= cmin) & (uc <= cmax)
        assert nd == len(uk) and no == int(keep.sum())
        assert np.array_equal(km, uk[keep]) and np.array_equal(ct, uc[keep].astype(np.uint32))
        # the allocating entry point
        with KmerCounter(k=31, p=11, partitions=1, counter="hash") as c:
            n2, d2 = c.count_keys(keys, cmin, cmax)
            k2, c2 = c.result()
        o2 = np.argsort(k2)
        assert (no, nd) == (n2, d2)
        assert np.array_equal(km, k2[o2]) and np.array_equal(ct, c2[o2])
    # limits: too many keys is refused before any work; a short output says how much is needed
    assert _noalloc(L, d_keys, (1 << 19) + 1, 1, U32, out_k, out_c, cap)[0] == GKC_ELIMIT
    rc, no, nd = _noalloc(L, d_keys, 1 << 19, 1, U32, out_k, out_c, 1000)
    assert rc == GKC_ELIMIT and no == nd and no > 1000
    # 5000 keys built to hash onto one slot: more than the probe limit, refused
    bad = np.array([_unhash(((i + 1) << 20) | 12345) for i in range(5000)], np.uint64)
    d_bad = torch.from_numpy(bad.view(np.int64)).to(dev)
    assert _noalloc(L, d_bad, len(bad), 1, U32, out_k, out_c, cap)[0] == GKC_ELIMIT
    # and the next call starts from a clear table
    rc, no, nd = _noalloc(L, d_bad, 3000, 1, U32, out_k, out_c, cap)
    assert rc == 0 and no == nd == 3000
    assert np.array_equal(np.sort(out_k[:no].cpu().numpy().view(np.uint64)), np.sort(bad[:3000]))
