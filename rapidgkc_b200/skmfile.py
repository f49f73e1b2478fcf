"""The reference's .skm partition files (skmstore.hpp:129-141): one file per
partition, `<folder><partition>.skm`, holding the partition's superkmers in
skm_3x bytes with no header (the reference keeps the counts in memory).

save_skm writes a counter's store this way (so the reference's phase 2, or a
later run of this counter, can count it); load_skm appends such files to a
counter's store, superkmer bounds and minimizers recovered on the GPU
(gkc_add_skm).  Files written by the reference's phase 1 load when the counter
uses the reference's k, p, partition count and the default order.
"""
from __future__ import annotations

import os

import numpy as np


def skm_path(folder: str, part: int) -> str:
    """The reference's name for partition `part`: PAR.tmp_file_folder + id + ".skm"."""
    return f"{folder}{part}.skm" if folder.endswith(os.sep) or not folder else os.path.join(folder, f"{part}.skm")


def save_skm(counter, folder: str) -> int:
    """Writes every partition of the counter's store; returns the bytes written."""
    os.makedirs(folder, exist_ok=True)
    total = 0
    for part in range(counter.partitions):
        data = counter.store_export(part)
        with open(skm_path(folder, part), "wb") as f:
            f.write(data.tobytes())
        total += len(data)
    return total


def load_skm(counter, folder: str) -> int:
    """Appends the partition files of `folder` (a missing file is an empty
    partition) to the counter's store as one chunk; returns the bytes read."""
    parts, off = [], np.zeros(counter.partitions + 1, np.uint64)
    for part in range(counter.partitions):
        path = skm_path(folder, part)
        data = np.fromfile(path, np.uint8) if os.path.exists(path) else np.zeros(0, np.uint8)
        parts.append(data)
        off[part + 1] = off[part] + len(data)
    if off[-1]:
        counter.add_skm(np.concatenate(parts), off)
    return int(off[-1])
