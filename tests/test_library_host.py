"""Host-side checks of libgpusketch_b200.so that need no GPU: it loads, exports every C-ABI symbol
of include/gpusketch.h, and its host functions agree with the oracle."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import gpusketch_b200 as gs
from gpusketch_b200 import _native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "gpusketch.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:gs_status|uint64_t|const char\*)\s+(gs_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    names = header_functions()
    assert len(names) >= 20
    L = _native.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_native.SIGNATURES), "ctypes signatures out of sync with the header"


def test_hash_matches_golden(golden_dir):
    for k, s, h in json.load(open(os.path.join(golden_dir, "xxh3_vectors.json"))):
        assert gs.hash64(int(k), int(s)) == int(h)


def test_geometry_matches_reference(golden_dir, restatement):
    for V, f, nb in json.load(open(os.path.join(golden_dir, "geometry.json"))):
        g = gs.geometry_for(V, f)
        assert g.num_buckets == nb and g.bytes_per_vertex == 16 * nb
        o = restatement.geometry(V, f)
        assert (g.num_samples, g.bkt_per_col) == (o["num_samples"], o["bkt_per_col"])


def test_geometry_rejects_bad_args():
    with pytest.raises(gs.GpuSketchError) as e:
        gs.geometry_for(1)
    assert e.value.status == _native.GS_ERR_BAD_ARG


def test_exact_min_cut_matches_stoer_wagner(restatement):
    rng = np.random.default_rng(1)
    for _ in range(150):
        V = int(rng.integers(2, 48))
        m = int(rng.integers(0, 160))
        e = rng.integers(0, V, size=(m, 2)).astype(np.uint32)
        v, side = gs.exact_min_cut(V, e)
        w, _ = restatement.stoer_wagner(V, e)
        assert v == w
        if 0 < side.sum() < V:
            assert sum(1 for a, b in e.tolist() if a != b and side[a] != side[b]) == v


def test_exact_min_cut_planted_blocks_vs_maxflow():
    """Two dense blocks joined by 3 edges: the global min cut is 3 (scipy max-flow cross-check)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import maximum_flow
    rng = np.random.default_rng(2)
    n = 60
    blocks = []
    for off in (0, n):
        a, b = np.triu_indices(n, 1)
        keep = rng.random(a.size) < 0.4
        blocks.append(np.stack([a[keep] + off, b[keep] + off], 1))
    cut = np.array([[1, n + 2], [5, n + 9], [7, n + 30]])
    e = np.concatenate(blocks + [cut]).astype(np.uint32)
    v, side = gs.exact_min_cut(2 * n, e)
    assert v == 3
    assert set(np.flatnonzero(side).tolist()) in (set(range(n)), set(range(n, 2 * n)))
    cap = csr_matrix((np.ones(2 * len(e), np.int32), (np.r_[e[:, 0], e[:, 1]], np.r_[e[:, 1], e[:, 0]])),
                     shape=(2 * n, 2 * n))
    assert maximum_flow(cap, 0, n).flow_value == 3


def test_er_stream_shape_and_determinism(restatement):
    a = gs.er_stream(1024, 0.05, 0x5EED0001, 0.10, 0.5)
    b = gs.er_stream(1024, 0.05, 0x5EED0001, 0.10, 0.5)
    assert np.array_equal(a, b)
    m = int(round(len(a) / 1.15))
    assert 24000 < m < 28500                      # ~ p * V(V-1)/2 = 26189 edges
    assert (a[:, 0] != a[:, 1]).all() and (a < 1024).all()
    final = restatement.final_edges(1024, a)
    assert abs(len(final) - 0.95 * m) < 10        # 10% deleted, half of those back


def test_rmat_stream_host_properties():
    r = gs.rmat_stream(12, 50000, 0x5EED0002)
    assert r.shape == (50000, 2) and (r < 4096).all() and (r[:, 0] != r[:, 1]).all()
    again = gs.rmat_stream(12, 1000, 0x5EED0002, first=1000)
    assert np.array_equal(again, r[1000:2000])    # counter-based: any slice regenerates exactly
    deg = np.bincount(r.reshape(-1), minlength=4096)
    assert deg[0] > 20 * np.median(deg)           # R-MAT skew: vertex 0 is a hub


def test_create_without_device_reports_no_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(gs.GpuSketchError) as e:
        gs.GraphSketch(1024, 1)
    assert e.value.status == _native.GS_ERR_NO_DEVICE
