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


# ── struct layouts: the header (compiled by a C compiler), the ctypes binding
#    and the Rust binding documented in INTEGRATION.md must agree byte for byte

def _c_layout(tmp_path, struct, fields):
    """sizeof and every field's offset of `struct` as gcc lays it out from
    include/polariseq_knn.h."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "polariseq_knn.h"',
             'int main(void) {', f'  printf("%zu\\n", sizeof({struct}));']
    lines += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines += ['  return 0;', '}']
    src = tmp_path / f"{struct}.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / struct
    subprocess.run([cc, "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return int(out[0]), [int(v) for v in out[1:]]


@pytest.mark.parametrize("struct,cls", [("pq_nnd_opts", _lib.NndOpts),
                                        ("pq_nnd_stats", _lib.NndStats)])
def test_ctypes_structs_match_the_header_layout(tmp_path, struct, cls):
    names = [f[0] for f in cls._fields_]
    size, offs = _c_layout(tmp_path, struct, names)
    assert C.sizeof(cls) == size, f"{struct}: ctypes {C.sizeof(cls)} bytes, C {size}"
    assert [getattr(cls, f).offset for f in names] == offs


def _rust_repr_c_layout(body):
    """Size and field offsets of a #[repr(C)] Rust struct body with scalar
    fields (the C layout rules: each field at the next multiple of its
    alignment, the size rounded up to the largest alignment)."""
    sizes = {"u64": 8, "i64": 8, "f64": 8, "u32": 4, "i32": 4, "f32": 4, "u8": 1, "i8": 1}
    fields = re.findall(r"pub\s+(\w+)\s*:\s*(\w+)", body)
    off, offs, align = 0, [], 1
    for name, ty in fields:
        s = sizes[ty]
        off = (off + s - 1) // s * s
        offs.append((name, off))
        off += s
        align = max(align, s)
    return (off + align - 1) // align * align, offs


def test_documented_rust_binding_matches_the_header(tmp_path):
    """The PqNndOpts struct a maintainer would paste from INTEGRATION.md has
    the header's field names, order, offsets and size."""
    doc = open(os.path.join(os.path.dirname(HEADER), "..", "INTEGRATION.md")).read()
    m = re.search(r"pub struct PqNndOpts\s*\{(.*?)\}", doc, flags=re.S)
    assert m, "no PqNndOpts in INTEGRATION.md"
    size, offs = _rust_repr_c_layout(m.group(1))
    names = [f[0] for f in _lib.NndOpts._fields_]
    assert [n for n, _ in offs] == names
    c_size, c_offs = _c_layout(tmp_path, "pq_nnd_opts", names)
    assert size == c_size
    assert [o for _, o in offs] == c_offs
