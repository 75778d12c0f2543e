"""Build recipe of the native libraries, in-tree (the built .so files travel with the repository).

  libbm25_b200.so   CUDA engine + C ABI (nvcc, sm_100a only)
  libbm25_synth.so  seeded synthetic corpus -> resident-index arrays (gcc + OpenMP)
  libbm25_facade.so C++ SDK facade (include/AscendIndexBm25.h) over the C ABI (g++)
  _hostcall*.so     Python entry points of the host-buffer Searches over the C ABI (gcc, CPython C API)

Run as ``python bm25-npu_b200/build.py`` or through ``__graft_entry__.build()``.
"""

import os
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / 'csrc'
INCLUDE = ROOT / 'include'
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']

ENGINE_SOURCES = ['engine.cu', 'mlp.cu', 'serve.cpp', 'builder.cu']
ENGINE_HEADERS = ['tile_kernels.cuh', 'stream_kernel.cuh', 'tile_group_kernel.cuh', 'warp_tile_kernel.cuh', 'block_kernels.cuh',
                  'block_tile_kernel.cuh',
                  'learned_kernels.cuh', 'mlp.cuh', 'merge_kernel.cuh']


def _stale(target, sources):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def _run(cmd):
    print(' '.join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_engine(force=False, verbose_ptxas=False):
    target = PACKAGE / 'libbm25_b200.so'
    sources = [CSRC / s for s in ENGINE_SOURCES]
    deps = sources + [CSRC / h for h in ENGINE_HEADERS] + [INCLUDE / 'bm25_b200.h', Path(__file__)]
    if not force and not _stale(target, deps):
        return target
    cmd = [NVCC, *ARCH, '-lineinfo', '-O3', '-std=c++17', '-shared', '-Xcompiler', '-fPIC,-fopenmp',
           '-I', INCLUDE, '-I', CSRC, '-o', target, *sources, '-lgomp']
    if verbose_ptxas:
        cmd[1:1] = ['-Xptxas', '-v']
    _run(cmd)
    return target


def build_synth(force=False):
    target = PACKAGE / 'libbm25_synth.so'
    src = CSRC / 'synth.c'
    if not force and not _stale(target, [src, Path(__file__)]):
        return target
    _run(['gcc', '-O3', '-std=c11', '-fopenmp', '-ffp-contract=off', '-fno-fast-math', '-fPIC', '-shared',
          '-o', target, src, '-lm'])
    return target


def build_facade(force=False):
    target = PACKAGE / 'libbm25_facade.so'
    src = CSRC / 'AscendIndexBm25.cpp'
    engine = build_engine(force)
    deps = [src, INCLUDE / 'AscendIndexBm25.h', INCLUDE / 'bm25_b200.h', engine, Path(__file__)]
    if not force and not _stale(target, deps):
        return target
    _run(['g++', '-O2', '-std=c++17', '-fPIC', '-shared', '-Wall', '-I', INCLUDE, '-o', target, src,
          '-L', PACKAGE, '-lbm25_b200', "-Wl,-rpath,$ORIGIN"])
    return target


def build_runner(force=False):
    """bm25_runner: the reference's benchmark runner command line on this engine (csrc/runner.cpp)."""
    target = PACKAGE / 'bm25_runner'
    src = CSRC / 'runner.cpp'
    engine = build_engine(force)
    deps = [src, INCLUDE / 'bm25_b200.h', engine, Path(__file__)]
    if not force and not _stale(target, deps):
        return target
    _run(['g++', '-O2', '-std=c++17', '-Wall', '-I', INCLUDE, '-I', '/usr/local/cuda/include', '-o', target, src,
          '-L', PACKAGE, '-lbm25_b200', '-L', '/usr/local/cuda/lib64', '-lcudart', "-Wl,-rpath,$ORIGIN"])
    return target


def build_hostcall(force=False):
    """_hostcall: the Python entry points of the host-buffer Searches (csrc/hostcall.c, CPython C API)."""
    import sysconfig
    target = PACKAGE / ('_hostcall' + sysconfig.get_config_var('EXT_SUFFIX'))
    src = CSRC / 'hostcall.c'
    engine = build_engine(force)
    deps = [src, INCLUDE / 'bm25_b200.h', engine, Path(__file__)]
    if not force and not _stale(target, deps):
        return target
    _run(['gcc', '-O2', '-std=c11', '-fPIC', '-shared', '-Wall', '-I', sysconfig.get_paths()['include'], '-I', INCLUDE,
          '-o', target, src, '-L', PACKAGE, '-lbm25_b200', "-Wl,-rpath,$ORIGIN"])
    return target


def build_all(force=False):
    return (build_engine(force), build_synth(force), build_facade(force), build_runner(force),
            build_hostcall(force))


if __name__ == '__main__':
    build_all(force='--force' in sys.argv)
