"""RapidGKC's own command-line program on the B200 library: the reference's
gkc_main.cpp and cpu_funcs.cpp with its two GPU files (gpu_skmgen.cu,
gpu_kmercounting.cu) replaced by the C++ shim of the integration guide
(rapidgkc_b200/shim/gkc_b200_shim.cpp), linked by oracle/Makefile into
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


def test_integration_guide_shows_the_committed_shim():
    """The shim in INTEGRATION.md is the file that is compiled."""
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    i = doc.index("```cpp\n// gkc_b200_shim.cpp")
    j = doc.index("```", i + 6)
    assert doc[i + 7:j] == open(SHIM).read()


@pytest.mark.gpu
@pytest.mark.parametrize("k,p,P", [(31, 11, 64), (25, 9, 31)])
def test_reference_main_through_the_shim(oracle, tmp_path, k, p, P):
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
    p_ = subprocess.run([BIN, "-gpuonly", "-ngpu", "1", "-im", "-t", "4", "-t2", "2", "-k", str(k), "-p", str(p),
                         "-skm", str(P), "-read", str(fq)], cwd=tmp_path, capture_output=True, text=True,
                        timeout=300)
    out = p_.stdout + p_.stderr
    assert p_.returncode == 0, out[-2000:]
    assert int(re.search(r"Total number of distinct kmers: (\d+)", out).group(1)) == do
    assert int(re.search(r"KMER TOT CNT = (\d+)", out).group(1)) == int(np.sum(pk))
