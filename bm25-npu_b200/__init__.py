"""B200-native BM25 Search engine: resident index in HBM, fused sm_100a scoring + top-K kernels.

Import with ``importlib.import_module('bm25-npu_b200')`` (the directory name is not
a Python identifier).  The CUDA engine (libbm25_b200.so) must be built in-tree
(``python bm25-npu_b200/build.py``); without it the Search API raises ImportError.
"""

from . import _native, autotune, learned, serving, sharded
from .corpus import (CONFIG_SHAPES, INDEX_FILES, CorpusSpec, LazyIndex, build_index, read_bm25s_dir, read_index_dir,
                     read_queries_dir, synthetic_index, synthetic_queries, unpack_queries, write_bm25s_dir,
                     write_index_dir, write_queries_dir)
from .search import (APP_ERR_ILLEGAL_OPERATION, APP_ERR_INNER_ERROR, APP_ERR_INVALID_PARAM, APP_ERR_OK,
                     AscendIndexBm25, Bm25Config, Bm25Error, Bm25SearchResult, Bm25Session, IllegalOperation,
                     InnerError, InvalidParam, pack_queries)

__all__ = [
    'CONFIG_SHAPES', 'INDEX_FILES', 'CorpusSpec', 'LazyIndex', 'build_index', 'read_index_dir', 'synthetic_index',
    'synthetic_queries', 'unpack_queries', 'write_index_dir', 'read_queries_dir', 'write_queries_dir',
    'read_bm25s_dir', 'write_bm25s_dir', 'APP_ERR_ILLEGAL_OPERATION', 'APP_ERR_INNER_ERROR',
    'APP_ERR_INVALID_PARAM', 'APP_ERR_OK', 'AscendIndexBm25', 'Bm25Config', 'Bm25Error', 'Bm25SearchResult',
    'Bm25Session', 'IllegalOperation', 'InnerError', 'InvalidParam', 'pack_queries', '_native', 'autotune', 'learned', 'serving', 'sharded',
]
