"""The allocation-free exact kNN entry point, through the C ABI (GPU).

`pq_neighbors_into_device_noalloc` is for callers that must not allocate
device memory themselves or have a library do it for them: a framework that
owns the whole device budget through its own memory pool, or a serving loop
where cudaMalloc / cudaFree would synchronise the device and stall other
streams.  It keeps its only scratch (the cosine metric's row norms) in a fixed
array inside the library.  These checks compare it with the context-based
`pq_neighbors_into_device` on the same inputs: the results must be identical
(the exact search is bit-exact, so the tolerance is zero), on two calls in a
row and after a larger call has left its own contents in the shared array.
This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""

import ctypes as C

import numpy as np
import pytest

import polariseq_b200 as pq
from polariseq_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _outs(torch, n, k):
    kws = min(k, n)
    m = max(n * (kws - 1), 1)
    return (torch.full((n + 1,), -1, dtype=torch.int32, device="cuda"),
            torch.full((m,), -1, dtype=torch.int32, device="cuda"),
            torch.full((m,), float("nan"), dtype=torch.float32, device="cuda"))


def _noalloc(torch, x, k, metric, stream=None):
    n, d = x.shape
    ip, ix, dx = _outs(torch, n, k)
    nnz = C.c_uint64(0)
    rc = _lib.load().pq_neighbors_into_device_noalloc(
        x.data_ptr(), n, d, k, pq.METRICS[metric], ip.data_ptr(), ix.data_ptr(), dx.data_ptr(),
        C.byref(nnz), None if stream is None else C.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, int(nnz.value), ip, ix, dx


def _with_context(torch, x, k, metric):
    n = x.shape[0]
    ip, ix, dx = _outs(torch, n, k)
    nnz = pq.default_context(0).neighbors_device(x, k, pq.METRICS[metric], ip, ix, dx)
    torch.cuda.synchronize()
    return nnz, ip, ix, dx


def _same(a, b):
    (nnz_a, ip_a, ix_a, dx_a), (nnz_b, ip_b, ix_b, dx_b) = a, b
    assert nnz_a == nnz_b
    assert torch_equal(ip_a, ip_b) and torch_equal(ix_a[:nnz_a], ix_b[:nnz_b])
    assert dx_a[:nnz_a].cpu().numpy().tobytes() == dx_b[:nnz_b].cpu().numpy().tobytes()


def torch_equal(a, b):
    return bool((a.cpu() == b.cpu()).all())


@pytest.mark.parametrize("metric", ["cosine", "euclidean"])
def test_matches_context_entry_point_twice(metric):
    torch = pytest.importorskip("torch")
    big = torch.from_numpy(synth.mixture_dirichlet(4000, 50, 12, seed=21)).cuda()
    small = torch.from_numpy(synth.mixture_dirichlet(1001, 13, 6, seed=22)).cuda()
    for x, k in ((big, 15), (small, 31)):  # the small call follows the big one's leftovers
        want = _with_context(torch, x, k, metric)
        for _ in range(2):
            rc, nnz, ip, ix, dx = _noalloc(torch, x, k, metric)
            assert rc == _lib.PQ_OK
            _same((nnz, ip, ix, dx), want)


def test_on_a_caller_stream():
    torch = pytest.importorskip("torch")
    x = torch.from_numpy(synth.mixture_dirichlet(2500, 50, 8, seed=23)).cuda()
    want = _with_context(torch, x, 15, "cosine")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        rc, nnz, ip, ix, dx = _noalloc(torch, x, 15, "cosine", stream=s.cuda_stream)
    assert rc == _lib.PQ_OK
    _same((nnz, ip, ix, dx), want)


def test_rejects_beyond_its_limits():
    """Each rejected call returns its code and leaves *nnz_out untouched."""
    torch = pytest.importorskip("torch")
    too_many = torch.zeros((262_145, 1), dtype=torch.float32, device="cuda")
    x = torch.zeros((10, 3), dtype=torch.float32, device="cuda")
    wide = torch.zeros((10, 513), dtype=torch.float32, device="cuda")
    for data, k, want in ((too_many, 2, _lib.PQ_ETOOBIG), (x, 0, _lib.PQ_EINVAL),
                          (x[:0], 5, _lib.PQ_EINVAL), (wide, 5, _lib.PQ_ENOTSUP)):
        rc, nnz = _noalloc(torch, data, k, "euclidean")[:2]
        assert rc == want
        assert nnz == 0


def test_accepts_exactly_its_row_limit():
    """262,144 rows fill the fixed norm array to its last element: accepted,
    and equal to the context path."""
    torch = pytest.importorskip("torch")
    g = np.random.default_rng(24)
    x = torch.from_numpy(g.standard_normal((262_144, 2)).astype(np.float32)).cuda()
    want = _with_context(torch, x, 3, "cosine")
    rc, nnz, ip, ix, dx = _noalloc(torch, x, 3, "cosine")
    assert rc == _lib.PQ_OK
    _same((nnz, ip, ix, dx), want)
