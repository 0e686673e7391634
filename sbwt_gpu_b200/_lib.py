"""ctypes binding of libsbwt_gpu.so (the C ABI declared in include/sbwt_gpu.h).

The shared library is built in-tree by ``sbwt_gpu_b200.build.build()``; importing
this module fails loudly if it is missing -- there is no pure-Python or CPU
fallback for any entry point.
"""
import ctypes
import os
from ctypes import POINTER, c_char_p, c_int, c_int32, c_int64, c_uint32, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
# SBWT_GPU_LIBRARY names another build of the same library (for example one
# compiled with different build options); the in-tree build otherwise.
LIB_PATH = os.environ.get("SBWT_GPU_LIBRARY") or os.path.join(HERE, "libsbwt_gpu.so")
CLI_PATH = os.path.join(HERE, "sbwt_search")

SBWT_POPPY = 1
SBWT_CUM_POPPY = 2
SBWT_LAYOUT_LINES = 0
SBWT_LAYOUT_POPPY = 1
SBWT_LAYOUT_LINES512 = 2
SBWT_LAYOUT_LINES2048 = 3


class Params(ctypes.Structure):
    """Mirror of ``sbwt_params`` (include/sbwt_gpu.h)."""

    _fields_ = [
        ("k", c_uint32),
        ("k_presearch", c_uint32),
        ("bits_in_superblock", c_uint32),
        ("rank_structure", c_int32),
        ("with_shuffles", c_int32),
        ("threads_per_block", c_uint32),
        ("device", c_int32),
        ("layout", c_int32),
        ("kmers_per_thread", c_uint32),
        ("threads_per_kmer", c_uint32),
        ("search_mode", c_int32),
    ]


class Queries(ctypes.Structure):
    """Mirror of ``sbwt_queries``."""

    _fields_ = [
        ("letters", POINTER(ctypes.c_uint8)),
        ("n_letters", c_uint64),
        ("row_starts", POINTER(c_uint64)),
        ("n_rows", c_uint64),
        ("n_kmers", c_uint64),
    ]


class Built(ctypes.Structure):
    """Mirror of ``sbwt_built``."""

    _fields_ = [
        ("n_bits", c_uint64),
        ("n_kmers", c_uint64),
        ("n_dummies", c_uint64),
        ("bits", POINTER(c_uint64) * 4),
        ("n_words", c_uint64),
    ]


class Profile(ctypes.Structure):
    """Mirror of ``sbwt_profile``."""

    _fields_ = [
        ("pack_ms", ctypes.c_float),
        ("table_ms", ctypes.c_float),
        ("search_ms", ctypes.c_float),
        ("member_ms", ctypes.c_float),
        ("launches", c_uint32),
        ("search_blocks", c_uint32),
    ]


class MlpParams(ctypes.Structure):
    """Mirror of ``sbwt_mlp_params``."""

    _fields_ = [
        ("steps", c_uint32),
        ("batch", c_uint32),
        ("lr", ctypes.c_float),
        ("n_positive", c_uint64),
        ("n_negative", c_uint64),
        ("seed", c_uint64),
        ("tau", ctypes.c_float),
        ("bloom_fpr", ctypes.c_float),
        ("bloom_hashes", c_uint32),
    ]


class PrefilterStats(ctypes.Structure):
    """Mirror of ``sbwt_prefilter_stats``."""

    _fields_ = [
        ("first_loss", ctypes.c_float),
        ("final_loss", ctypes.c_float),
        ("train_ms", ctypes.c_float),
        ("total_ms", ctypes.c_float),
        ("n_train", c_uint64),
        ("label_positive_fraction", ctypes.c_double),
        ("train_accuracy", ctypes.c_double),
        ("n_indexed_kmers", c_uint64),
        ("n_rejected_indexed", c_uint64),
        ("bloom_bits", c_uint64),
    ]


# name -> (restype, argtypes): every symbol include/sbwt_gpu.h declares
SIGNATURES = {
    "sbwt_params_default": (c_int, [POINTER(Params)]),
    "sbwt_last_error": (c_char_p, []),
    "sbwt_index_load": (c_int, [c_char_p, c_char_p, c_char_p, c_char_p, POINTER(Params), POINTER(c_void_p)]),
    "sbwt_index_from_host": (c_int, [POINTER(c_void_p), c_uint64, POINTER(Params), POINTER(c_void_p)]),
    "sbwt_index_free": (None, [c_void_p]),
    "sbwt_index_info": (c_int, [c_void_p, POINTER(c_uint64), POINTER(c_uint64), POINTER(c_uint32), POINTER(c_uint32)]),
    "sbwt_presearch": (c_int, [c_void_p, c_uint32]),
    "sbwt_build_times": (c_int, [c_void_p, POINTER(ctypes.c_float)]),
    "sbwt_pipeline_bytes": (c_int, [c_void_p, POINTER(ctypes.c_uint64), POINTER(ctypes.c_uint64)]),
    "sbwt_presearch_export": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64]),
    "sbwt_rank_export": (c_int, [c_void_p, c_uint32, c_int32, c_int, c_void_p, c_uint64, c_void_p, c_uint64]),
    "sbwt_configure": (c_int, [c_void_p, c_int32, c_uint32, c_int32, c_int32, c_uint32, c_uint32, c_uint32]),
    "sbwt_set_search_mode": (c_int, [c_void_p, c_int32]),
    "sbwt_node_bytes_export": (c_int, [c_void_p, c_void_p, c_uint64]),
    "sbwt_search_packed": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, c_void_p]),
    "sbwt_pack": (c_int, [c_void_p, c_uint64, c_void_p, c_void_p]),
    "sbwt_search_reads": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, c_void_p, c_void_p, c_uint64,
                                  c_void_p]),
    "sbwt_search_reads_noalloc": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, c_void_p, c_void_p,
                                          c_uint64, c_void_p]),
    "sbwt_search_reads_host": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, c_void_p, c_uint64]),
    "sbwt_search_reads_host_member": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, c_void_p, c_uint64]),
    "sbwt_count_kmers": (c_uint64, [c_void_p, c_uint64, c_uint32]),
    "sbwt_profile_enable": (c_int, [c_void_p, c_int]),
    "sbwt_use_graphs": (c_int, [c_void_p, c_int]),
    "sbwt_set_l2_fetch_granularity": (c_int, [c_void_p, c_uint32]),
    "sbwt_profile_read": (c_int, [c_void_p, POINTER(Profile)]),
    "sbwt_mlp_params_default": (c_int, [POINTER(MlpParams)]),
    "sbwt_prefilter_train": (c_int, [c_void_p, POINTER(MlpParams), POINTER(c_void_p)]),
    "sbwt_prefilter_stats_get": (c_int, [c_void_p, POINTER(PrefilterStats)]),
    "sbwt_prefilter_params": (c_int, [c_void_p, c_void_p, c_uint64]),
    "sbwt_prefilter_free": (None, [c_void_p]),
    "sbwt_prefilter_logits": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_void_p]),
    "sbwt_search_kmers": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_void_p]),
    "sbwt_search_kmers_filtered": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_void_p, POINTER(c_uint64),
                                           c_void_p]),
    "sbwt_search_reads_host_multi": (c_int, [c_void_p, c_int, c_void_p, c_uint64, c_void_p, c_uint64, c_void_p,
                                             c_uint64]),
    "sbwt_partition_rows": (c_int, [c_void_p, c_uint64, c_uint32, c_int, c_void_p]),
    "sbwt_set_walk_options": (c_int, [c_void_p, c_uint32, c_uint32, c_int32, c_int32]),
    "sbwt_set_host_threads": (c_int, [c_void_p, c_int]),
    "sbwt_pipeline_dense_share": (ctypes.c_double, [c_uint64, c_int]),
    "sbwt_search_reads_filtered": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, c_void_p,
                                           c_void_p, c_uint64, POINTER(c_uint64), c_void_p]),
    "sbwt_mlp_gradients": (c_int, [c_uint32, c_void_p, c_void_p, c_void_p, c_uint32, POINTER(ctypes.c_float),
                                   c_void_p]),
    "sbwt_mlp_logits": (c_int, [c_uint32, c_void_p, c_void_p, c_uint64, c_void_p]),
    "sbwt_queries_read": (c_int, [c_char_p, c_uint32, POINTER(Queries)]),
    "sbwt_queries_read_many": (c_int, [POINTER(c_char_p), c_int, c_uint32, POINTER(Queries), c_void_p]),
    "sbwt_autotune": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_uint64, c_uint64, c_void_p, c_uint32, c_void_p,
                              c_uint64]),
    "sbwt_queries_free": (None, [POINTER(Queries)]),
    "sbwt_reader_open": (c_int, [c_char_p, c_uint32, POINTER(c_void_p)]),
    "sbwt_reader_next": (c_int, [c_void_p, c_uint64, POINTER(Queries)]),
    "sbwt_reader_close": (None, [c_void_p]),
    "sbwt_format_answers": (c_int64, [c_void_p, c_uint64, c_uint32, c_void_p, c_void_p, c_uint64]),
    "sbwt_build": (c_int, [c_void_p, c_void_p, c_uint64, c_uint32, POINTER(Built)]),
    "sbwt_format_answers_device": (c_int, [c_void_p, c_uint64, c_uint32, c_void_p, c_uint64, c_void_p, c_uint64,
                                           POINTER(c_uint64), c_void_p]),
    "sbwt_build_gpu": (c_int, [c_void_p, c_void_p, c_uint64, c_uint32, c_int32, POINTER(Built)]),
    "sbwt_build_free": (None, [POINTER(Built)]),
    "sbwt_write_bitvector": (c_int, [c_char_p, c_void_p, c_uint64]),
}


def load_library(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(this engine has no fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load_library()


class SbwtError(RuntimeError):
    """A C-ABI call returned non-zero; the message is sbwt_last_error()."""


def check(rc):
    if rc != 0:
        raise SbwtError(lib.sbwt_last_error().decode(errors="replace"))
    return rc
