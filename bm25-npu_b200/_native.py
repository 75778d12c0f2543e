"""ctypes bindings of the engine's C ABI (include/bm25_b200.h).

The engine library is loaded from this package directory only; if it is
missing the import fails loudly -- there is no CPU or Python fallback.
"""

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_uint32, c_uint64, c_void_p
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ENGINE_PATH = PACKAGE / 'libbm25_b200.so'
SYNTH_PATH = PACKAGE / 'libbm25_synth.so'

BM25_OK = 0
BM25_ERR_INVALID_PARAM = 1
BM25_ERR_ILLEGAL_OPERATION = 2
BM25_ERR_INNER_ERROR = 3
BM25_INJECT_HOST_FAILURE = 1
BM25_INJECT_STALL = 2


class ServerOptions(ctypes.Structure):
    _fields_ = [
        ('max_batch', c_int32),
        ('learned', c_int32),
        ('max_wait_us', c_int32),
        ('reserved', c_int32),
        ('candidate_budget', c_int64),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ('device_id', c_int32),
        ('max_k', c_int32),
        ('query_capacity', c_int64),
        ('word_capacity', c_int64),
        ('tile_docs', c_int32),
        ('merge_fan_in', c_int32),
        ('directory_bytes', c_int64),
        ('stream', c_void_p),
        ('kernel', c_int32),
        ('ring_stages', c_int32),
        ('ring_chunk', c_int32),
        ('prune', c_int32),
        ('candidate_capacity', c_int64),
        ('prune_route', c_float),
        ('wait_budget_cycles', c_int64),
        ('dense_density', c_float),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [
        ('claim_tiles', c_int32),
        ('tail_claims', c_int32),
        ('ring_stages', c_int32),
        ('ring_chunk', c_int32),
        ('candidate_cap', c_int64),
        ('prune_route', c_float),
        ('reserved', c_int32),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ('num_docs', c_int64),
        ('vocab', c_int64),
        ('postings', c_int64),
        ('tile_docs', c_int32),
        ('tiles', c_int32),
        ('merge_fan_in', c_int32),
        ('merge_levels', c_int32),
        ('directory_rows', c_int64),
        ('directory_min_df', c_int64),
        ('index_bytes', c_int64),
        ('device_bytes', c_int64),
        ('graph_replays', c_int64),
        ('searches', c_int64),
        ('kernel', c_int32),
        ('ring_stages', c_int32),
        ('grid', c_int32),
        ('smem_bytes', c_int32),
        ('ring_chunk', c_int32),
        ('query_capacity', c_int32),
        ('word_capacity', c_int32),
        ('max_k', c_int32),
        ('prune', c_int32),
        ('graph_instantiations', c_int64),
        ('graphs_cached', c_int64),
        ('dense_rows', c_int64),
    ]


# Every symbol include/bm25_b200.h declares, with its ctypes signature.
SIGNATURES = {
    'bm25_default_options': (None, [POINTER(Options)]),
    'bm25_create': (c_int, [POINTER(c_int64), POINTER(c_int32), POINTER(c_float), c_int64, c_int64,
                            POINTER(Options), POINTER(c_void_p)]),
    'bm25_create_lazy': (c_int, [POINTER(c_int64), POINTER(c_int32), POINTER(c_float), POINTER(c_float),
                                 POINTER(c_float), c_int64, c_int64, c_float, POINTER(Options), POINTER(c_void_p)]),
    # the per-Search call takes plain addresses (numpy's .ctypes.data): no pointer objects on the hot path
    'bm25_search': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p]),
    'bm25_search_device': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p]),
    'bm25_device_status': (c_int, [c_void_p, POINTER(c_uint32)]),
    'bm25_close': (c_int, [c_void_p]),
    'bm25_destroy': (None, [c_void_p]),
    'bm25_last_error': (c_int, [c_void_p, c_char_p, c_size_t, POINTER(c_int64)]),
    'bm25_get_info': (c_int, [c_void_p, POINTER(Info)]),
    'bm25_kernel_timing': (c_int, [c_void_p, c_int32]),
    'bm25_test_inject': (c_int, [c_void_p, c_int32]),
    'bm25_prepare_batch_graphs': (c_int, [c_void_p, c_int32, c_int32]),
    'bm25_get_tuning': (c_int, [c_void_p, POINTER(Tuning)]),
    'bm25_set_tuning': (c_int, [c_void_p, POINTER(Tuning)]),
    'bm25_kernel_times': (c_int, [c_void_p, POINTER(c_float), c_int64, POINTER(c_int64)]),
    'bm25_search_pruned_device': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p,
                                          c_void_p, c_void_p, c_void_p]),
    'bm25_search_pruned': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p,
                                   c_void_p]),
    'bm25_search_batch': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    'bm25_search_batch_learned': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p,
                                          c_void_p]),
    'bm25_search_batch_device': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_int32,
                                         c_void_p, c_void_p, c_void_p, c_void_p]),
    'bm25_merge_topk': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_int32, c_int64, c_int32,
                                c_void_p, c_void_p, c_void_p]),
    'bm25_default_server_options': (None, [c_void_p]),
    'bm25_server_create': (c_int, [c_void_p, c_void_p, c_void_p]),
    'bm25_server_submit': (c_int, [c_void_p, c_void_p, c_int32, c_int32, c_void_p]),
    'bm25_server_wait': (c_int, [c_void_p, c_uint64, c_void_p, c_void_p, c_void_p, c_void_p]),
    'bm25_server_stats': (c_int, [c_void_p, c_void_p, c_void_p]),
    'bm25_server_destroy': (c_int, [c_void_p]),
    'bm25_server_last_error': (c_int, [c_void_p, c_size_t]),
    'bm25_serve_poisson': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_double, c_int64,
                                   c_uint64, c_void_p, c_void_p, c_void_p]),
    'bm25_build_index': (c_int, [c_void_p, c_void_p, c_int64, c_int64, c_double, c_double, c_int32, c_void_p,
                                 c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    'bm25_build_last_error': (c_int, [c_void_p, c_size_t]),
    'bm25_set_threshold_model': (c_int, [c_void_p, c_void_p, c_float]),
    'bm25_query_features_device': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p,
                                           c_void_p]),
    'bm25_search_learned': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p]),
    'bm25_search_learned_device': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p,
                                           c_void_p, c_void_p]),
    'bm25_search_stats': (c_int, [c_void_p, c_void_p, c_int32]),
    'bm25_mlp_param_count': (c_int64, []),
    'bm25_mlp_scratch_floats': (c_int64, [c_int64]),
    'bm25_mlp_forward': (c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    'bm25_mlp_gradient': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_float, c_void_p, c_void_p, c_void_p,
                                  c_void_p]),
    'bm25_mlp_adam': (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_int32, c_void_p]),
    'bm25_mlp_last_error': (c_int, [ctypes.c_char_p, c_size_t]),
    'bm25_search_csc_static': (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_int64,
                                       c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_int32]),
}

_engine = None


def engine_library():
    """Loads libbm25_b200.so from this package, or raises ImportError."""
    global _engine
    if _engine is None:
        if not ENGINE_PATH.exists():
            raise ImportError(f'BM25 CUDA engine not built: {ENGINE_PATH} is missing (run bm25-npu_b200/build.py)')
        lib = ctypes.CDLL(str(ENGINE_PATH))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _engine = lib
    return _engine


_hostcall = None


def hostcall():
    """The host-buffer Search entry points over the buffer protocol (_hostcall, built beside the
    engine), or ImportError."""
    global _hostcall
    if _hostcall is None:
        engine_library()  # the engine first, from this package
        import importlib
        try:
            _hostcall = importlib.import_module(__package__ + '._hostcall')
        except ImportError as e:
            raise ImportError(f'BM25 host call module not built in {PACKAGE} (run bm25-npu_b200/build.py): {e}')
    return _hostcall


_synth = None


def synth_library():
    global _synth
    if _synth is None:
        if not SYNTH_PATH.exists():
            raise ImportError(f'Synthetic corpus library not built: {SYNTH_PATH} is missing')
        lib = ctypes.CDLL(str(SYNTH_PATH))
        lib.synth_create.restype = c_void_p
        lib.synth_create.argtypes = [c_int64, c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_uint64, c_int]
        lib.synth_postings.restype = c_int64
        lib.synth_postings.argtypes = [c_void_p]
        lib.synth_tokens.restype = c_int64
        lib.synth_tokens.argtypes = [c_void_p]
        lib.synth_fill.restype = c_int
        lib.synth_fill.argtypes = [c_void_p, ctypes.c_double, ctypes.c_double, POINTER(c_int64), POINTER(c_int32),
                                   POINTER(c_float), POINTER(c_float), POINTER(c_float), POINTER(c_int32)]
        lib.synth_destroy.restype = None
        lib.synth_destroy.argtypes = [c_void_p]
        lib.synth_queries.restype = c_int64
        lib.synth_queries.argtypes = [POINTER(c_int64), c_int64, c_int64, c_int32, c_int32, c_int, ctypes.c_uint64,
                                      POINTER(c_int64), POINTER(c_int32)]
        _synth = lib
    return _synth


def ptr(array, ctype):
    """Pointer to a C-contiguous numpy array's data."""
    return array.ctypes.data_as(POINTER(ctype))
