"""The C-ABI library without a GPU: it loads, exports every symbol that
include/polariseq_knn.h declares, and the host-side argument handling mirrors
the reference binding (crates/polariseq-python/src/lib.rs:503-566)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

import polariseq_b200 as pq
from polariseq_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "polariseq_knn.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pq_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    syms = declared_symbols()
    assert syms, "no declarations parsed"
    for s in syms:
        assert hasattr(L, s), f"{s} declared in the header but not exported"
    assert set(syms) == set(_lib.EXPORTS)


def test_effective_k_matches_the_reference():
    for n, k, want in [(1, 15, 1), (5, 10, 4), (100, 15, 15), (16, 15, 15), (2, 0, 1)]:
        assert pq.effective_k(n, k) == want


def test_default_options_mirror_nndescent_options_default():
    o = _lib.NndOpts()
    _lib.load().pq_nnd_opts_default(C.byref(o))
    assert (o.k, o.max_candidates, o.max_iterations, o.n_trees, o.leaf_size, o.gather_max,
            o.seed) == (15, 0, 0, 0, 0, 0, 0)
    assert o.delta == pytest.approx(0.001)


def test_out_arrays_are_validated_before_any_device_work():
    emb = np.zeros((10, 3), np.float32)
    with pytest.raises(ValueError, match="11 row pointers and 90 neighbours"):
        pq.nndescent_dense(emb, 9, out=(np.zeros(10, np.uint32), np.zeros(90, np.uint32),
                                        np.zeros(90, np.float32)))
    with pytest.raises(ValueError):
        pq.nndescent_dense(emb, 9, out=(np.zeros(11, np.uint32), np.zeros(89, np.uint32),
                                        np.zeros(90, np.float32)))
    with pytest.raises(TypeError):
        pq.nndescent_dense(emb, 9, out=(np.zeros(11, np.int64), np.zeros(90, np.uint32),
                                        np.zeros(90, np.float32)))


def test_panicking_inputs_raise_panic_exception():
    with pytest.raises(pq.PanicException):
        pq.nndescent_dense(np.zeros((0, 3), np.float32), 5)
    with pytest.raises(pq.PanicException):
        pq.nndescent_dense(np.zeros((10, 3), np.float32), 0)
    assert not issubclass(pq.PanicException, Exception)


def test_embedding_type_checks():
    with pytest.raises(TypeError):
        pq.nndescent_dense(np.zeros((10, 3), np.float64), 5)
    with pytest.raises(TypeError):
        pq.nndescent_dense(np.zeros(10, np.float32), 5)


def test_null_context_and_args_are_rejected_without_a_device():
    L = _lib.load()
    o = _lib.NndOpts()
    L.pq_nnd_opts_default(C.byref(o))
    nnz = C.c_uint64()
    assert L.pq_nndescent_into(None, None, 10, 3, C.byref(o), None, 11, None, 0, None, 0,
                               C.byref(nnz)) == _lib.PQ_EINVAL
    assert L.pq_ctx_last_error(None) == b"null context"
