"""Host helpers of bench.py (CPU): the FASTQ the reference program reads in
the reference arm holds exactly the sampled reads."""
import numpy as np
import pytest

from oracle.fastx_oracle import parse_fastx
from tests_util import random_reads


@pytest.mark.parametrize("lens", [150, (31, 300)])
def test_write_fastq_round_trips(tmp_path, lens):
    import bench
    reads, offs = random_reads(41, 50_000, 500, lens, 0.01)
    path = tmp_path / "s.fq"
    bench.write_fastq(str(path), reads, offs)
    got, state = parse_fastx(path.read_bytes(), "fastq")
    assert state == 0
    exp = [reads[int(offs[i]):int(offs[i + 1])].tobytes() for i in range(len(offs) - 1)]
    assert got == exp
