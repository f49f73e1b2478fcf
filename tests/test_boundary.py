"""The boundary in five calls (gkc_init, gkc_skmgen_batch,
gkc_count_partition, gkc_set_order_lut, gkc_shutdown): the reference's GPU
interface step by step (GPUReset, GenSuperkmerGPU per batch, then
kmc_counting_GPU_streams per store), through ctypes, against the oracle."""
import ctypes as C

import numpy as np
import pytest

from tests_util import random_reads

U32 = 0xFFFFFFFF


def _lib():
    from rapidgkc_b200.capi import load_library
    return load_library()


def test_null_context_is_rejected_without_a_device():
    from rapidgkc_b200.capi import GKC_EINVAL, Options
    L = _lib()
    o = Options()
    L.gkc_default_options(C.byref(o))
    o.k = 65  # beyond the 128-bit build's 64: rejected before any device call
    h = C.c_void_p()
    assert L.gkc_init(0, C.byref(o), C.byref(h)) == GKC_EINVAL
    assert L.gkc_shutdown(None) == GKC_EINVAL
    assert L.gkc_set_order_lut(None, None) == GKC_EINVAL
    no, nd = C.c_uint64(), C.c_uint64()
    assert L.gkc_count_partition(None, 0, 1, U32, None, None, 0, 0, C.byref(no), C.byref(nd)) == GKC_EINVAL
    assert L.gkc_skmgen_batch(None, None, None, 0, 31, 11, 512, None, 0, None, None, None) == GKC_EINVAL


@pytest.mark.gpu
@pytest.mark.parametrize("counter,order", [("sort", False), ("hash", True)])
def test_five_calls_match_the_oracle(oracle, counter, order):
    from rapidgkc_b200.capi import COUNTER_HASH, COUNTER_SORT, GKC_EINVAL, GKC_ESTATE, GKC_OK, MEM_HOST, Options
    L = _lib()
    k, p, P = 31, 11, 16
    reads, offs = random_reads(21, 40_000, 3000, (20, 300), 0.005)
    lut = np.random.default_rng(22).permutation(4 ** p).astype(np.uint32) if order else None
    pbo, pso, pko, _, _ = oracle.skmgen(reads, offs, k, p, P, lut)
    ko, co, do, _ = oracle.count_reads(reads, offs, k, p, P, 2, U32, lut)
    o = Options()
    L.gkc_default_options(C.byref(o))
    o.k, o.p, o.partitions = k, p, P
    o.counter = COUNTER_SORT if counter == "sort" else COUNTER_HASH
    h = C.c_void_p()
    assert L.gkc_init(0, C.byref(o), C.byref(h)) == GKC_OK
    try:
        pb, ps, pk = (np.zeros(P, np.uint64) for _ in range(3))
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        # two batches, as the reference's loader hands GenSuperkmerGPU one batch at a time
        half = (len(offs) - 1) // 2
        batches = [(reads, offs[:half + 1]), (reads[int(offs[half]):], offs[half:] - offs[half])]
        lut_p = ptr(lut) if order else None
        assert L.gkc_skmgen_batch(h, ptr(batches[0][0]), ptr(batches[0][1]), half, k, p + 1, P, None, MEM_HOST,
                                  None, None, None) == GKC_EINVAL  # p must be the context's
        for i, (r, of) in enumerate(batches):
            rc = L.gkc_skmgen_batch(h, ptr(r), ptr(np.ascontiguousarray(of, np.uint64)), len(of) - 1, k, p, P,
                                    lut_p if i == 0 else None, MEM_HOST, ptr(pb), ptr(ps), ptr(pk))
            assert rc == GKC_OK
        if order:  # the order of a non-empty store is fixed
            assert L.gkc_skmgen_batch(h, ptr(reads), ptr(offs), 0, k, p, P, lut_p, MEM_HOST, None, None,
                                      None) == GKC_ESTATE
        assert np.array_equal(pb, pbo) and np.array_equal(ps, pso) and np.array_equal(pk, pko)
        ks, cs, dist = [], [], 0
        for part in range(P):
            cap = int(pk[part]) + 1
            km = np.zeros(cap, np.uint64)
            ct = np.zeros(cap, np.uint32)
            no, nd = C.c_uint64(), C.c_uint64()
            assert L.gkc_count_partition(h, part, 2, U32, ptr(km), ptr(ct), cap, MEM_HOST, C.byref(no),
                                         C.byref(nd)) == GKC_OK
            ks.append(km[:no.value])
            cs.append(ct[:no.value])
            dist += nd.value
        km, ct = np.concatenate(ks), np.concatenate(cs)
        if counter == "hash":  # unordered inside a partition: compare partition by partition, sorted
            o1, o2 = np.lexsort((km,)), np.lexsort((ko,))
            assert np.array_equal(np.sort(km), np.sort(ko))
            assert np.array_equal(ct[o1], co[o2])
        else:  # partition by partition, ascending within: the oracle's order
            assert np.array_equal(km, ko) and np.array_equal(ct, co)
        assert dist == do
        assert L.gkc_set_order_lut(h, None) == GKC_OK  # back to the default order
    finally:
        assert L.gkc_shutdown(h) == GKC_OK


def _build_c_example(tmp_path):
    """Compiles the plain-C example (rapidgkc_b200/examples/five_calls.c) as
    C11 with every warning an error; returns the program's path."""
    import os
    import subprocess
    from conftest import ROOT
    src = os.path.join(ROOT, "rapidgkc_b200", "examples", "five_calls.c")
    exe = tmp_path / "five_calls"
    lib = os.path.join(ROOT, "rapidgkc_b200")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), "-o",
                    str(exe), src, "-L", lib, "-lrapidgkc_b200", f"-Wl,-rpath,{lib}"], check=True,
                   capture_output=True, timeout=120)
    return str(exe)


def test_c_example_compiles_as_c11(tmp_path):
    import subprocess
    import torch
    exe = _build_c_example(tmp_path)
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU test runs the program")
    p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert p.returncode == 1 and "gkc_init" in p.stderr  # no device here: refused, no CPU fallback


@pytest.mark.gpu
def test_c_example_counts_match_the_oracle(oracle, tmp_path):
    import subprocess
    exe = _build_c_example(tmp_path)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    r0 = b"ACGTTGCAAGGCTTACCGATGCATGCAAGTCCGATTAGCCGATAGGCTAACGTTAGC"
    r1 = b"TTGACCGTAGGCATCGATCGGATCCAAGTTGCAGCATGCAACGTTGCAAGGCTTACCGATG"
    reads = np.frombuffer(r0 + r1, np.uint8).copy()
    offs = np.array([0, len(r0), len(r0) + len(r1)], np.uint64)
    _, _, d, pk = oracle.count_reads(reads, offs, 31, 11, 4, 1)
    assert p.stdout.split() == ["instances", str(int(pk.sum())), "distinct", str(d)]
