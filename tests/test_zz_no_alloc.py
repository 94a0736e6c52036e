"""naga_knn_noalloc: the kNN search for callers that cannot allocate device
memory while they run (a fixed memory budget handed to their own allocator,
or a latency-critical path where cudaMalloc could stall other streams). It
keeps its scratch in one device array inside the library, so these checks
call it through the C ABI, twice in a row on different clouds, and compare
with the allocating naga_knn, which must agree bit for bit (the kNN bar of
this library). Collected last so a failure here leaves the rest of the GPU
suite already run; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(naga, src, qry, k):
    import torch

    s = torch.from_numpy(src).cuda()
    q = torch.from_numpy(qry).cuda()
    idx = torch.empty((len(qry), k), dtype=torch.int32, device="cuda")
    d2 = torch.empty((len(qry), k), dtype=torch.float32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = naga.lib().naga_knn_noalloc(C.c_void_p(s.data_ptr()), len(src), C.c_void_p(q.data_ptr()), len(qry),
                                     src.shape[1], k, C.c_void_p(idx.data_ptr()), C.c_void_p(d2.data_ptr()),
                                     stream)
    torch.cuda.synchronize()
    return rc, idx.cpu().numpy(), d2.cpu().numpy()


def _reference(naga, src, qry, k):
    import torch

    idx, d2 = naga.knn(torch.from_numpy(src).cuda(), torch.from_numpy(qry).cuda(), k)
    torch.cuda.synchronize()
    return idx.cpu().numpy(), d2.cpu().numpy()


def test_knn_noalloc_matches_knn_on_two_calls_in_a_row(naga):
    rng = np.random.default_rng(11)
    cases = [
        (rng.random((40000, 3)).astype(np.float32), rng.random((5000, 3)).astype(np.float32), 32),
        (rng.random((3000, 2)).astype(np.float32), (rng.random((800, 2)) * 1.2 - 0.1).astype(np.float32), 16),
    ]
    for src, qry, k in cases:
        rc, idx, d2 = _noalloc(naga, src, qry, k)
        assert rc == naga.NAGA_OK, naga.lib().naga_last_error()
        ri, rd = _reference(naga, src, qry, k)
        assert np.array_equal(idx, ri)
        assert np.array_equal(d2, rd)


def test_knn_noalloc_rejects_clouds_beyond_its_scratch(naga):
    src = np.zeros((65537, 3), np.float32)
    qry = np.zeros((1, 3), np.float32)
    rc, _, _ = _noalloc(naga, src, qry, 4)
    assert rc == naga.NAGA_EINVAL
    assert b"65536" in naga.lib().naga_last_error()


def test_knn_noalloc_rejects_nonfinite_coordinates(naga):
    """A NaN or infinite source coordinate is an input error found at the
    bounding box, before the search runs; the next call is unaffected."""
    rng = np.random.default_rng(12)
    src = rng.random((3000, 3)).astype(np.float32)
    qry = rng.random((50, 3)).astype(np.float32)
    for bad in (np.nan, np.inf, -np.inf):
        s = src.copy()
        s[17, 2] = bad
        rc, _, _ = _noalloc(naga, s, qry, 8)
        assert rc == naga.NAGA_EINVAL
        assert b"non-finite" in naga.lib().naga_last_error()
    rc, idx, d2 = _noalloc(naga, src, qry, 8)
    assert rc == naga.NAGA_OK
    ri, rd = _reference(naga, src, qry, 8)
    assert np.array_equal(idx, ri) and np.array_equal(d2, rd)


def test_knn_noalloc_edge_cases_match_knn(naga):
    """The cases that take the allocation-free search's own paths, each
    compared with naga_knn bit for bit: a 3-D cloud on a plane (its flat
    bounding box makes the first cell grid far larger than the fixed
    scratch, so the cells are coarsened), k = 64 (two list registers per
    lane), exactly 65,536 source points (the scratch's limit) and an empty
    cloud with queries (every slot the sentinel)."""
    rng = np.random.default_rng(13)
    plane = rng.random((40000, 3)).astype(np.float32)
    plane[:, 2] = 0.5
    slab = rng.random((20000, 3)).astype(np.float32)
    slab[:, 1] *= 1e-3
    full = rng.random((65536, 3)).astype(np.float32)
    cases = [
        (plane, rng.random((3000, 3)).astype(np.float32), 32),
        (slab, rng.random((2000, 3)).astype(np.float32), 16),
        (rng.random((5000, 3)).astype(np.float32), rng.random((1500, 3)).astype(np.float32), 64),
        (full, rng.random((4000, 3)).astype(np.float32), 32),
        (full[:, :2].copy(), rng.random((4000, 2)).astype(np.float32), 48),
    ]
    for src, qry, k in cases:
        rc, idx, d2 = _noalloc(naga, src, qry, k)
        assert rc == naga.NAGA_OK, naga.lib().naga_last_error()
        ri, rd = _reference(naga, src, qry, k)
        assert np.array_equal(idx, ri), (src.shape, k)
        assert np.array_equal(d2, rd), (src.shape, k)
    empty = np.zeros((0, 3), np.float32)
    qry = rng.random((10, 3)).astype(np.float32)
    rc, idx, d2 = _noalloc(naga, empty, qry, 8)
    assert rc == naga.NAGA_OK
    assert (idx.view(np.uint32) == 0xFFFFFFFF).all() and np.isinf(d2).all()
