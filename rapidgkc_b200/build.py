"""Builds the native libraries in-tree (they travel with the source tree).

    python -m rapidgkc_b200.build          # everything
    python -m rapidgkc_b200.build --ptxas  # also print register/spill usage

Outputs (git-ignored):
    rapidgkc_b200/librapidgkc_b200.so   CUDA kernels + C ABI (sm_100a only)
    rapidgkc_b200/libgkc_synth.so       seeded synthetic read generator
    rapidgkc_b200/gkc_main              command-line front end
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def _csrc(*names):
    return [os.path.join(CSRC, n) for n in names]


def build_cuda(ptxas: bool = False, force: bool = False) -> str:
    out = os.path.join(PKG, "librapidgkc_b200.so")
    srcs = [os.path.join(CSRC, n) for n in sorted(os.listdir(CSRC)) if n.endswith((".cu", ".cuh"))]
    srcs += [os.path.join(CSRC, "pack_host.cpp"), os.path.join(ROOT, "include", "gkc_capi.h")]
    if force or ptxas or _stale(out, srcs):
        # engine.cu includes the other .cu files; pack_host.cpp is host code
        # (its AVX2 path is chosen at run time)
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
               "-Xcompiler", "-fPIC", "-shared", "-o", out, os.path.join(CSRC, "engine.cu"),
               os.path.join(CSRC, "pack_host.cpp")]
        if ptxas:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd)
    return out


def build_synth(force: bool = False) -> str:
    out = os.path.join(PKG, "libgkc_synth.so")
    src = os.path.join(CSRC, "synth.cpp")
    if force or _stale(out, [src]):
        _run(["g++", "-std=c++17", "-O3", "-fPIC", "-shared", "-pthread", "-o", out, src])
    return out


def build_cli(force: bool = False) -> str:
    out = os.path.join(PKG, "gkc_main")
    src = os.path.join(CSRC, "gkc_main.cpp")
    lib = build_cuda()
    if os.path.exists(src) and (force or _stale(out, [src, lib])):
        cuda = os.path.dirname(os.path.dirname(NVCC))
        _run(["g++", "-std=c++17", "-O2", "-o", out, src, "-I", os.path.join(ROOT, "include"),
              "-I", os.path.join(cuda, "include"), "-L", PKG, "-lrapidgkc_b200", "-L", os.path.join(cuda, "lib64"),
              "-lcudart", "-lz", "-Wl,-rpath,$ORIGIN", "-pthread"])
    return out


def build_oracle(ref_tree: str | None = None) -> None:
    """The test oracles (oracle/Makefile).  The reference part is built only
    when the reference source tree is given (`ref_tree`, or the environment
    variable GKC_REFERENCE_TREE) and exists; otherwise the prebuilt
    oracle/_ref files are used as they are."""
    oracle = os.path.join(ROOT, "oracle")
    _run(["make", "-s", "-C", oracle, "liboracle.so"])
    ref_tree = ref_tree or os.environ.get("GKC_REFERENCE_TREE")
    if ref_tree and os.path.isdir(ref_tree):
        _run(["make", "-s", "-C", oracle, "ref", f"REF={ref_tree}"])


def build_all(ptxas: bool = False, force: bool = False, ref_tree: str | None = None) -> None:
    build_cuda(ptxas=ptxas, force=force)
    build_synth(force=force)
    build_cli(force=force)
    build_oracle(ref_tree)


if __name__ == "__main__":
    build_all(ptxas="--ptxas" in sys.argv, force="--force" in sys.argv)
