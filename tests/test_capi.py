"""The C ABI library: it loads, exports every symbol include/gkc_capi.h
declares, and refuses to run without a CUDA device (no CPU fallback).
No compute is called here."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gkc_capi.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gkc_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from rapidgkc_b200.capi import EXPORTS, load_library
    lib = load_library()
    syms = declared_symbols()
    assert len(syms) >= 15
    assert sorted(EXPORTS) == syms
    for s in syms:
        assert hasattr(lib, s), s


def test_errors_and_defaults_without_device():
    from rapidgkc_b200.capi import GKC_EINVAL, Options, load_library
    lib = load_library()
    o = Options()
    lib.gkc_default_options(ctypes.byref(o))
    assert (o.k, o.p, o.partitions) == (31, 11, 512)
    assert lib.gkc_strerror(GKC_EINVAL) == b"invalid argument"
    h = ctypes.c_void_p()
    o.p = 2  # out of range: rejected before any device call
    assert lib.gkc_create(0, ctypes.byref(o), ctypes.byref(h)) == GKC_EINVAL


def test_counter_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from rapidgkc_b200 import GkcError, KmerCounter
    with pytest.raises(GkcError):
        KmerCounter()
