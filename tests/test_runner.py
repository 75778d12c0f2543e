"""bm25_runner: the reference's benchmark runner command line (benchmark.cpp:31-110) on this engine.

CPU: usage and input errors end with status 1 before any device work.  GPU: on
the reference-built 2048-doc index (golden files written in the reference's
layout), the runner's checkpoints equal the original-document oracle's strict
top-K bit for bit, and its session record holds every measured sample.
"""

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
RUNNER = ROOT / 'bm25-npu_b200' / 'bm25_runner'
GOLDEN = Path(__file__).resolve().parent / 'golden'


@pytest.fixture(scope='module')
def runner(pkg):
    sys_build = __import__('importlib').import_module('bm25-npu_b200.build')
    sys_build.build_runner()
    return RUNNER


def _raw(path, offsets, words):
    rows = [words[offsets[i]:offsets[i + 1]] for i in range(offsets.size - 1)]
    text = f'BM25_QUERY_IDS_V1 {len(rows)}\n' + '\n'.join(' '.join(str(w) for w in [len(r), *r]) for r in rows)
    path.write_text(text + '\n')


def test_runner_rejects_bad_arguments(runner, tmp_path):
    r = subprocess.run([str(runner)], capture_output=True, text=True)
    assert r.returncode == 1 and 'Usage' in r.stderr
    bad = tmp_path / 'bad.txt'
    bad.write_text('NOT_A_QUERY_FILE 1\n')
    args = [str(runner), str(tmp_path), str(bad), str(bad), str(tmp_path / 'out'), '0', '-', '10', '8', '24', '1',
            '10', str(bad), str(bad)]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 1 and 'raw query ID file header' in r.stderr


@pytest.mark.gpu
def test_runner_on_reference_index(runner, tmp_path, cuda_ok):
    z = np.load(GOLDEN / 'large_corpus_n2048.npz')
    idx = tmp_path / 'index'
    idx.mkdir()
    z['offsets'].astype('<i8').tofile(idx / 'term_offsets.bin')
    z['docs'].astype('<i4').tofile(idx / 'posting_doc_ids.bin')
    z['tf'].astype('<f4').tofile(idx / 'posting_tf.bin')
    z['norm'].astype('<f4').tofile(idx / 'doc_norm.bin')
    z['idf'].astype('<f4').tofile(idx / 'idf.bin')
    for case in ('A', 'B'):
        _raw(tmp_path / f'{case}.txt', z[f'{case}_offsets'], z[f'{case}_words'])
        z[f'{case}_expected_scores'].astype('<f4').tofile(tmp_path / f'{case}_expected.bin')
    out = tmp_path / 'run'
    args = [str(runner), str(idx), str(tmp_path / 'A.txt'), str(tmp_path / 'B.txt'), str(out), '0', 'none', '10',
            '8', '24', '2', '10', str(tmp_path / 'A_expected.bin'), str(tmp_path / 'B_expected.bin')]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    for cp, case in (('before_A', 'A'), ('before_B', 'B'), ('after_A', 'A'), ('after_B', 'B')):
        ids = np.fromfile(out / cp / 'top_ids.bin', dtype='<i4').reshape(8, 10)
        scores = np.fromfile(out / cp / 'top_scores.bin', dtype='<f4').reshape(8, 10)
        assert np.array_equal(ids, z[f'{case}_top_ids'])
        assert np.array_equal(scores.view(np.uint32), z[f'{case}_top_scores'].view(np.uint32))
        assert json.loads((out / cp / 'check.json').read_text())['mismatched_queries'] == 0
    rec = json.loads((out / 'benchmark_session.json').read_text())
    assert rec['backend'] == 'b200' and rec['measured_search_calls'] == 20 and len(rec['samples']) == 20
    assert all(s['call_wall_ms'] > 0 for s in rec['samples'])
    mem = tmp_path / 'mem.json'
    assert subprocess.run([str(runner), '--memory', '0', str(mem)]).returncode == 0
    m = json.loads(mem.read_text())
    assert 0 < m['free'] <= m['total']
