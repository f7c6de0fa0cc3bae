"""ctypes binding of the C ABI in include/polariseq_knn.h.

Loading fails loudly: there is no CPU fallback anywhere in this package.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpq_knn.so")

PQ_OK, PQ_EINVAL, PQ_ENOMEM, PQ_EDEVICE, PQ_ETIMEOUT, PQ_ENOTSUP, PQ_ETOOBIG = range(7)
PQ_MODE_PLAIN, PQ_MODE_BF16, PQ_MODE_FP8 = 0, 1, 2
PQ_INIT_RP, PQ_INIT_LEARNED = 0, 1
PQ_METRIC_EUCLIDEAN, PQ_METRIC_COSINE = 0, 1
PQ_BATCH_AUTOTUNE, PQ_BATCH_GRAPH = 1, 2

# Every symbol include/polariseq_knn.h declares.
EXPORTS = (
    "pq_nnd_opts_default", "pq_effective_k", "pq_ctx_create", "pq_ctx_destroy",
    "pq_ctx_last_error", "pq_ctx_stats", "pq_nndescent_into", "pq_nndescent_into_device",
    "pq_nndescent_probe", "pq_debug_tree", "pq_ctx_set_profiling", "pq_neighbors_into",
    "pq_neighbors_into_device", "pq_neighbors_into_device_noalloc", "pq_knn_batched_into_device",
    "pq_mlp_params", "pq_mlp_grad", "pq_fuzzy_connectivities", "pq_fuzzy_connectivities_device",
    "pq_ctx_set_test_wait", "pq_scrublet_scores_device",
)


class NndOpts(C.Structure):
    """pq_nnd_opts: mirrors NndescentOptions (nndescent.rs:42-76)."""

    _fields_ = [
        ("k", C.c_uint64),
        ("max_candidates", C.c_uint64),
        ("max_iterations", C.c_uint64),
        ("delta", C.c_double),
        ("n_trees", C.c_uint64),
        ("leaf_size", C.c_uint64),
        ("gather_max", C.c_uint64),
        ("seed", C.c_uint64),
        ("mode", C.c_int32),
        ("init", C.c_int32),
        ("probes", C.c_int32),
        ("refine_rounds", C.c_int32),
        ("buckets", C.c_int32),
    ]


class NndStats(C.Structure):
    _fields_ = [
        ("rounds_run", C.c_int32),
        ("n_trees", C.c_int32),
        ("k", C.c_uint64),
        ("max_candidates", C.c_uint64),
        ("n_iters", C.c_uint64),
        ("leaf_size", C.c_uint64),
        ("stop_at", C.c_uint64),
        ("changed", C.c_uint64 * 64),
        ("emitted", C.c_uint64 * 64),
        ("pairs", C.c_uint64 * 64),
        ("ms_forest", C.c_double),
        ("ms_leaves", C.c_double),
        ("ms_rounds", C.c_double),
        ("ms_extract", C.c_double),
        ("ms_total", C.c_double),
        ("launches", C.c_uint64),
        ("kg_ms", C.c_double * 16),
        ("kg_launches", C.c_uint64 * 16),
        ("shortlist", C.c_uint64 * 8),
        ("learn_loss_first", C.c_double),
        ("learn_loss_last", C.c_double),
        ("ms_learn_train", C.c_double),
        ("ms_learn_route", C.c_double),
        ("est_recall", C.c_double),
        ("est_recall_learned", C.c_double),
        ("est_recall_rp", C.c_double),
        ("fell_back", C.c_int32),
        ("learned_rounds", C.c_int32),
    ]


KERNEL_GROUPS = ("forest_top", "seqtree", "leaf_pairs", "candidates", "join_count",
                 "join_write", "sort", "replay", "extract", "buckets", "layout", "tiles",
                 "rerank")


_lib = None
_lock = threading.Lock()


def load(build_if_missing: bool = False):
    """Load the in-tree sm_100a library; raises if it is absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            if build_if_missing:
                from . import build as _b

                _b.build()
            else:
                raise RuntimeError(
                    f"polariseq_b200: CUDA library not built ({LIB_PATH}); run "
                    "`python -m polariseq_b200.build` (there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        U64 = C.c_uint64
        L.pq_nnd_opts_default.argtypes = [C.POINTER(NndOpts)]
        L.pq_nnd_opts_default.restype = None
        L.pq_effective_k.argtypes = [U64, U64]
        L.pq_effective_k.restype = U64
        L.pq_ctx_create.argtypes = [C.c_int, C.POINTER(P)]
        L.pq_ctx_create.restype = C.c_int
        L.pq_ctx_destroy.argtypes = [P]
        L.pq_ctx_destroy.restype = None
        L.pq_ctx_last_error.argtypes = [P]
        L.pq_ctx_last_error.restype = C.c_char_p
        L.pq_ctx_stats.argtypes = [P, C.POINTER(NndStats)]
        L.pq_ctx_stats.restype = C.c_int
        L.pq_ctx_set_profiling.argtypes = [P, C.c_int]
        L.pq_ctx_set_profiling.restype = C.c_int
        L.pq_ctx_set_test_wait.argtypes = [P, C.c_uint32]
        L.pq_ctx_set_test_wait.restype = C.c_int
        L.pq_nndescent_into.argtypes = [P, P, U64, U64, C.POINTER(NndOpts), P, U64, P, U64, P,
                                        U64, C.POINTER(U64)]
        L.pq_nndescent_into.restype = C.c_int
        L.pq_nndescent_into_device.argtypes = [P, P, U64, U64, C.POINTER(NndOpts), P, P, P,
                                               C.POINTER(U64), P]
        L.pq_nndescent_into_device.restype = C.c_int
        L.pq_nndescent_probe.argtypes = [P, P, U64, U64, C.POINTER(NndOpts), C.c_int32, P, P,
                                         P, P, P]
        L.pq_nndescent_probe.restype = C.c_int
        L.pq_debug_tree.argtypes = [P, P, U64, U64, C.POINTER(NndOpts), C.c_uint32, P, P, U64,
                                    C.POINTER(U64)]
        L.pq_debug_tree.restype = C.c_int
        L.pq_neighbors_into.argtypes = [P, P, U64, U64, U64, C.c_int32, P, U64, P, U64, P, U64,
                                         C.POINTER(U64)]
        L.pq_neighbors_into.restype = C.c_int
        L.pq_neighbors_into_device.argtypes = [P, P, U64, U64, U64, C.c_int32, P, P, P,
                                                C.POINTER(U64), P]
        L.pq_neighbors_into_device.restype = C.c_int
        L.pq_neighbors_into_device_noalloc.argtypes = [P, U64, U64, U64, C.c_int32, P, P, P,
                                                        C.POINTER(U64), P]
        L.pq_neighbors_into_device_noalloc.restype = C.c_int
        L.pq_knn_batched_into_device.argtypes = [P, P, U64, C.c_uint32, P, P, P, P, C.c_int32,
                                                  C.POINTER(C.c_int32), P]
        L.pq_knn_batched_into_device.restype = C.c_int
        L.pq_mlp_params.argtypes = [U64]
        L.pq_mlp_params.restype = U64
        L.pq_mlp_grad.argtypes = [P, U64, P, P, U64, P, P, C.c_uint32, P, P, P]
        L.pq_mlp_grad.restype = C.c_int
        L.pq_fuzzy_connectivities.argtypes = [P, U64, P, P, P, P, P, P, U64, C.POINTER(U64)]
        L.pq_fuzzy_connectivities.restype = C.c_int
        L.pq_fuzzy_connectivities_device.argtypes = [P, U64, P, P, P, U64, P, P, P, U64,
                                                     C.POINTER(U64), P]
        L.pq_fuzzy_connectivities_device.restype = C.c_int
        L.pq_scrublet_scores_device.argtypes = [P, C.c_uint32, U64, P, P, P, P, P, P, P, P,
                                                C.c_double, P, P, P, P, P, P]
        L.pq_scrublet_scores_device.restype = C.c_int
        _lib = L
        return L
