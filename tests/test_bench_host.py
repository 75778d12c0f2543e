"""Host-side helpers of bench.py (no device needed)."""

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402

from helpers import pack  # noqa: E402


def test_split_queries_rebuilds_the_set():
    rng = np.random.default_rng(3)
    rows = [[int(x) for x in rng.integers(0, 1000, int(rng.integers(0, 11)))] for _ in range(1003)]
    offsets, words = pack(rows)
    ks = rng.choice([10, 100], len(rows)).astype(np.int32)
    parts = bench.split_queries(offsets, words, ks, 250)
    assert [p[2].size for p in parts] == [250, 250, 250, 250, 3]
    got_rows = [list(p[1][p[0][i]:p[0][i + 1]]) for p in parts for i in range(p[0].size - 1)]
    assert got_rows == rows
    assert np.array_equal(np.concatenate([p[2] for p in parts]), ks)
    for qo, w, _ in parts:
        assert qo.dtype == np.int64 and qo[0] == 0 and qo[-1] == w.size
