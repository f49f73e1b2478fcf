"""Shared fixtures.  `-m "not gpu"` runs on any machine; `-m gpu` needs a
CUDA device (B200) and the in-tree librapidgkc_b200.so."""
import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built CUDA library")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle.oracle import RefOracle
    try:
        return RefOracle()
    except FileNotFoundError as e:
        pytest.skip(str(e))


@pytest.fixture(scope="session")
def ref_oracle_wide():
    """The reference's 128-bit LONGERKMER build, for k > 32."""
    from oracle.oracle import RefOracle
    try:
        return RefOracle(wide=True)
    except FileNotFoundError as e:
        pytest.skip(str(e))


def golden_cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


def split_superkmers(stream):
    """Superkmers of a partition stream: first byte, full bytes, terminal
    non-full byte (cpu_funcs.cpp:238-244)."""
    out, i, n = [], 0, len(stream)
    while i < n:
        j = i + 1
        while j < n and (stream[j] >> 6) == 3:
            j += 1
        out.append(bytes(stream[i:j + 1]))
        i = j + 1
    return out


def partition_digest(stream):
    import hashlib
    h = hashlib.sha256()
    for s in sorted(split_superkmers(stream)):
        h.update(len(s).to_bytes(4, "little"))
        h.update(s)
    return h.hexdigest()


def sorted_table(kmers, counts):
    """The table in ascending k-mer order (u64 keys, or (n, 2) low/high pairs
    ordered as 128-bit values for k > 32)."""
    if kmers.ndim == 2:
        o = np.lexsort((kmers[:, 0], kmers[:, 1]))
    else:
        o = np.argsort(kmers, kind="stable")
    return kmers[o], counts[o]
