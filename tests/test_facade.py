"""The C++ SDK facade (include/AscendIndexBm25.h) driven by a compiled C++ test program."""

import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from helpers import assert_same_topk

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / 'bm25-npu_b200'


@pytest.fixture(scope='module')
def facade_bin(tmp_path_factory, pkg):
    import importlib
    build = importlib.import_module('bm25-npu_b200.build')
    build.build_facade()
    exe = tmp_path_factory.mktemp('facade') / 'facade_test'
    subprocess.run(['g++', '-O1', '-std=c++17', '-Wall', '-I', str(ROOT / 'include'), '-o', str(exe),
                    str(ROOT / 'tests' / 'cpp' / 'facade_test.cpp'), '-L', str(PKG), '-lbm25_facade', '-lbm25_b200',
                    f'-Wl,-rpath,{PKG}'], check=True)
    return exe


def test_facade_lifecycle_and_input_errors(facade_bin):
    r = subprocess.run([str(facade_bin), 'host'], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_facade_search_matches_oracle(facade_bin, pkg, oracle_mod, cuda_ok, tmp_path):
    spec = pkg.CONFIG_SHAPES['synthetic_8192']
    index = pkg.synthetic_index(spec)
    pkg.write_index_dir(index, tmp_path / 'index')
    offsets, words = pkg.synthetic_queries(index.offsets, 8, 3, 3, 4)
    k = 10
    bits = struct.unpack('<i', struct.pack('<f', spec.k1))[0]
    header = np.array([offsets.size - 1, k, bits], dtype=np.int64)
    with open(tmp_path / 'queries.bin', 'wb') as f:
        f.write(header.tobytes() + offsets.astype(np.int64).tobytes() + words.astype(np.int32).tobytes())
    out = tmp_path / 'out.bin'
    r = subprocess.run([str(facade_bin), 'device', str(tmp_path / 'index'), str(tmp_path / 'queries.bin'), str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    q = offsets.size - 1
    raw = out.read_bytes()
    scores = np.frombuffer(raw[:q * k * 4], dtype=np.float32).reshape(q, k)
    labels = np.frombuffer(raw[q * k * 4:], dtype=np.int64).reshape(q, k)
    data = oracle_mod.contributions(index, spec.k1)
    ref = oracle_mod.search(index.offsets, index.docs, data, index.num_docs, offsets, words, k)
    assert_same_topk(scores, labels.astype(np.int32), *ref, 'facade')
