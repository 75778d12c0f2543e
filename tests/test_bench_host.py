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


def test_step_check_counts_every_step_on_cpu_tensors():
    """StepCheck copies each step's outputs into its own slot and compares them bit for bit after the
    loop (here on CPU tensors: the same code the bench runs on device tensors)."""
    import torch
    out = [torch.zeros(6, dtype=torch.float32), torch.zeros(6, dtype=torch.int32)]
    want = [(np.arange(6, dtype=np.float32), np.arange(6, dtype=np.int32)),
            (np.full(6, 2.5, np.float32), np.full(6, 7, np.int32))]
    check = bench.StepCheck(out, lambda i: want[i % 2], 4)
    for i in range(4):
        out[0].copy_(torch.from_numpy(want[i % 2][0]))
        out[1].copy_(torch.from_numpy(want[i % 2][1]))
        if i == 3:
            out[0][5] = float(np.nextafter(np.float32(2.5), np.float32(3)))  # one bit off
        check.capture(i)
    check.verify(4)
    assert check.report() == {'checked_searches': 4, 'mismatched': 1, 'bit_exact': False}


def test_step_check_compares_packed_prefixes_only():
    import torch
    out = [torch.full((8,), 9.0)]
    check = bench.StepCheck(out, lambda i: [np.array([1.0, 2.0, 3.0], np.float32)], 1, length=lambda i: 3)
    out[0][:3] = torch.tensor([1.0, 2.0, 3.0])
    check.capture(0)
    check.verify(1)
    assert check.report()['bit_exact']


def test_same_bits_and_algorithmic_bytes():
    a = (np.array([1.0, 0.0], np.float32), np.array([3, 4], np.int32))
    b = (np.array([1.0, -0.0], np.float32), np.array([3, 4], np.int32))
    assert bench.same_bits(a, a) and not bench.same_bits(a, b)  # -0.0 and +0.0 differ in bits
    df = np.array([10, 20, 30], np.int64)
    offsets, words = np.array([0, 2, 4], np.int64), np.array([0, 1, 1, 5], np.int32)  # word 5: out of vocabulary
    assert bench.algorithmic_bytes(df, 3, offsets, words, 10) == (10 + 20 + 20) * 8 + 3 * 16 + 2 * 10 * 8
    assert bench.algorithmic_bytes(df, 3, offsets, words, 10, distinct=True) == (10 + 20) * 8 + 2 * 16 + 2 * 10 * 8
