"""The allocation-free ingest entry point (gs_ingest_pairs_noalloc).

It exists for callers that cannot call cudaMalloc because another allocator owns the device memory
(a framework's caching allocator, an embedded runtime that forbids allocation after start-up): they
pass their own sketch buffer, and the library's scratch is a static device array.  This file is
collected last, so a stop at the first failure has run every other test first; it passes alone in a
fresh process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

import gpusketch_b200 as gs
from gpusketch_b200 import _native


def _call(V, seed, pairs_ptr, n, sk_ptr, factor=1.0):
    return _native.lib().gs_ingest_pairs_noalloc(V, seed, factor, C.c_void_p(pairs_ptr), n, C.c_void_p(sk_ptr), None)


def test_noalloc_rejects_sizes_beyond_its_maximum():
    L = _native.lib()
    assert _call(70000, 1, 0, 0, 1) == _native.GS_ERR_BAD_ARG
    assert b"num_vertices" in L.gs_last_error()
    assert _call(1000, 1, 1, 65537, 1) == _native.GS_ERR_BAD_ARG
    assert b"edge records" in L.gs_last_error()
    assert _call(1, 1, 1, 10, 1) == _native.GS_ERR_BAD_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("V,factor", [(50000, 1.0), (65536, 1.0), (65536, 1.5)])
def test_noalloc_matches_graph_ingest_on_two_calls(V, factor):
    """At the vertex limit with full 65536-record batches (every bucketing region at its largest), and
    with sketches_factor 1.5 (33 columns: two columns per lane), two calls in a row equal the existing
    entry point byte for byte."""
    import torch
    assert torch.cuda.is_available()
    seed = 0xABCDEF
    geo = gs.geometry_for(V, factor)
    assert (geo.num_columns > 32) == (factor > 1.0)
    nb = geo.num_buckets
    rng = np.random.default_rng(21 + V)
    hub = np.stack([np.full(9000, 7, np.uint32), rng.integers(0, V, 9000).astype(np.uint32)], 1)
    batches = [np.concatenate([rng.integers(0, V, size=(65536 - 9000, 2), dtype=np.uint32), hub]),
               rng.integers(0, V, size=(65536, 2), dtype=np.uint32)]
    batches[1][:4] = [[V - 1, 0], [V - 1, V - 2], [0, V - 1], [V - 2, V - 1]]   # the highest vertex ids
    sk = torch.zeros(V * nb * 2, dtype=torch.int64, device="cuda")   # the caller's own sketch buffer
    with gs.GraphSketch(V, seed, sketches_factor=factor) as g:
        for b in batches:
            g.ingest_pairs(b)                                        # the existing entry point
            d = torch.from_numpy(b.astype(np.int32)).cuda()
            torch.cuda.synchronize()
            rc = _call(V, seed, d.data_ptr(), len(b), sk.data_ptr(), factor)
            assert rc == _native.GS_OK, _native.lib().gs_last_error()
            assert sk.cpu().numpy().tobytes() == g.download().tobytes()   # bit-exact, as every test here
