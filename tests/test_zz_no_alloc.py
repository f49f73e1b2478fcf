"""gkc_count_keys_noalloc: the raw-key hash count with fixed device scratch
and no allocation, through the C ABI, against gkc_count_keys.  Collected last
on purpose; it must also pass alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

U32 = 0xFFFFFFFF


def _noalloc(L, d_keys, n, cmin, cmax, out_k, out_c, cap):
    no, nd = C.c_uint64(0), C.c_uint64(0)
    rc = L.gkc_count_keys_noalloc(C.c_void_p(d_keys.data_ptr()), n, cmin, cmax, C.c_void_p(out_k.data_ptr()),
                                  C.c_void_p(out_c.data_ptr()), cap, C.byref(no), C.byref(nd), None)
    return rc, no.value, nd.value


@pytest.mark.gpu
def test_noalloc_matches_count_keys_on_consecutive_calls():
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
        keys[keys == np.uint64(U32 << 32 | U32)] = 1
        d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
        rc, no, nd = _noalloc(L, d_keys, n, cmin, cmax, out_k, out_c, cap)
        assert rc == 0
        km = out_k[:no].cpu().numpy().view(np.uint64)
        ct = out_c[:no].cpu().numpy().view(np.uint32)
        o = np.argsort(km)
        with KmerCounter(k=31, p=11, partitions=1, counter="hash") as c:
            n2, d2 = c.count_keys(keys, cmin, cmax)
            k2, c2 = c.result()
        o2 = np.argsort(k2)
        assert (no, nd) == (n2, d2)
        assert np.array_equal(km[o], k2[o2]) and np.array_equal(ct[o], c2[o2])
    # limits: too many keys is refused before any work; a short output says how much is needed
    assert _noalloc(L, d_keys, (1 << 19) + 1, 1, U32, out_k, out_c, cap)[0] == GKC_ELIMIT
    rc, no, nd = _noalloc(L, d_keys, 1 << 19, 1, U32, out_k, out_c, 1000)
    assert rc == GKC_ELIMIT and no == nd and no > 1000
