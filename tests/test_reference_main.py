"""RapidGKC's own command-line program on the B200 library: the reference's
gkc_main.cpp and cpu_funcs.cpp with its two GPU files (gpu_skmgen.cu,
gpu_kmercounting.cu) replaced by the C++ shim
rapidgkc_b200/shim/gkc_b200_shim.cpp, linked by oracle/Makefile into
oracle/_ref/rapidgkc_on_b200 where the reference tree exists.  The program's
own report (distinct k-mers, k-mer instances) must equal the oracle's."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from tests_util import random_reads

BIN = os.path.join(ROOT, "oracle", "_ref", "rapidgkc_on_b200")
SHIM = os.path.join(ROOT, "rapidgkc_b200", "shim", "gkc_b200_shim.cpp")


@pytest.mark.gpu
@pytest.mark.parametrize("k,p,P,ngpu", [(31, 11, 64, 1), (25, 9, 31, 1), (31, 11, 64, 2), (21, 7, 37, 3)])
def test_reference_main_through_the_shim(oracle, tmp_path, k, p, P, ngpu):
    """-ngpu N: phase 1 takes devices round-robin and phase 2 counts each
    partition group on its worker's device after pulling the group's
    superkmers from the other devices.  With fewer GPUs than N, devices share
    a GPU (one context each), which runs the same mapping and exchange."""
    if not os.path.exists(BIN):
        pytest.skip(f"{BIN} not built (needs the reference tree: make -C oracle ref)")
    reads, offs = random_reads(77, 50_000, 20_000, 150, 0.003)
    fq = tmp_path / "reads.fq"
    with open(fq, "wb") as f:
        for i in range(len(offs) - 1):
            s = reads[int(offs[i]):int(offs[i + 1])].tobytes()
            f.write(b"@r%d\n%s\n+\n%s\n" % (i, s, b"I" * len(s)))
    _, _, do, pk = oracle.count_reads(reads, offs, k, p, P, 1)
    # -gpuonly: every batch goes through GenSuperkmerGPU; -im: stores in memory
    p_ = subprocess.run([BIN, "-gpuonly", "-ngpu", str(ngpu), "-tgpu", "1", "-im", "-t", "4", "-t2", str(max(2, ngpu)),
                         "-k", str(k), "-p", str(p), "-skm", str(P), "-rb", "3000", "-read", str(fq)], cwd=tmp_path,
                        capture_output=True, text=True, timeout=300)
    out = p_.stdout + p_.stderr
    assert p_.returncode == 0, out[-2000:]
    assert int(re.search(r"Total number of distinct kmers: (\d+)", out).group(1)) == do
    assert int(re.search(r"KMER TOT CNT = (\d+)", out).group(1)) == int(np.sum(pk))
