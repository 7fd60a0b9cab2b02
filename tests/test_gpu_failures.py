"""The failure statuses the C ABI promises, reached without faulting, trapping or hanging a GPU:
Boruvka running out of sketch columns (the reference's OutOfSamplesException, src/sketch.cpp:111-113)
and a bounded device-side wait that gives up (GS_ERR_TIMEOUT).  After either, the same handle answers
the next query correctly."""
import numpy as np
import pytest

import gpusketch_b200 as gs
from gpusketch_b200 import _native

pytestmark = pytest.mark.gpu


def _garbage_sketches(V, nb, seed):
    """Buckets whose every sample fails: a deterministic bucket that is neither zero nor good and no
    good bucket in any column (a random gamma equals XXH3(alpha) with probability 2^-64)."""
    rng = np.random.default_rng(seed)
    return rng.integers(1, 2**63, size=(V, nb * 2), dtype=np.uint64)


def test_out_of_samples_is_sketch_fail(restatement):
    V, seed = 700, 0x5EED4000
    with gs.GraphSketch(V, seed) as g:
        nb = g.geometry.num_buckets
        junk = _garbage_sketches(V, nb, 1)
        g.upload(junk.view(gs.BUCKET_DTYPE).reshape(V, nb))
        with pytest.raises(gs.GpuSketchError) as e:
            g.connected_components()
        assert e.value.status == _native.GS_ERR_SKETCH_FAIL
        assert b"ran out of samples" in _native.lib().gs_last_error()
        with pytest.raises(gs.GpuSketchError) as e:
            g.spanning_forest()
        assert e.value.status == _native.GS_ERR_SKETCH_FAIL
        # the restatement of the reference's Boruvka runs out of samples on the same sketches
        st, _, _, _ = restatement.boruvka(junk.reshape(-1).copy(), V, seed)
        assert st == -1
        # the handle is usable again once the sketches are valid
        g.clear()
        pairs = gs.er_stream(V, 0.004, 3, 0.1, 0.5)
        g.ingest_pairs(pairs)
        labels, ncc, _ = g.connected_components()
        n, exact = restatement.exact_cc(V, pairs)
        assert ncc == n and np.array_equal(labels, exact)


def test_out_of_samples_in_one_vertex_range_only(restatement):
    """Junk in a few vertices' sketches only: their components keep failing, so the query runs out of
    samples, as the reference's does."""
    V, seed = 1500, 0x5EED4001
    pairs = gs.er_stream(V, 0.003, 5, 0.1, 0.5)
    with gs.GraphSketch(V, seed) as g:
        g.ingest_pairs(pairs)
        good = g.download()
        nb = g.geometry.num_buckets
        g.upload(_garbage_sketches(4, nb, 2).view(gs.BUCKET_DTYPE).reshape(4, nb), first=100)
        with pytest.raises(gs.GpuSketchError) as e:
            g.connected_components()
        assert e.value.status == _native.GS_ERR_SKETCH_FAIL
        g.upload(good[100:104], first=100)
        labels, _, _ = g.connected_components()
        assert np.array_equal(labels, restatement.exact_cc(V, pairs)[1])


def test_grid_barrier_wait_gives_up_with_timeout(restatement):
    """A wait limit of one nanosecond makes the first block that waits at a grid barrier give up: the
    query returns GS_ERR_TIMEOUT, every block of the kernel returns, and with the default limit the same
    handle answers exactly."""
    V, seed = 1 << 16, 0x5EED4002
    pairs = gs.rmat_stream(16, 400_000, 0x5EED4003)
    with gs.GraphSketch(V, seed) as g:
        g.ingest_pairs(pairs)
        before = g.download()
        g.set_device_wait_limit(1)
        with pytest.raises(gs.GpuSketchError) as e:
            g.connected_components()
        assert e.value.status == _native.GS_ERR_TIMEOUT
        assert b"gave up" in _native.lib().gs_last_error()
        g.set_device_wait_limit(0)                      # the default limit again
        labels, ncc, _ = g.connected_components()
        n, exact = restatement.exact_cc(V, pairs)
        assert ncc == n and np.array_equal(labels, exact)
        assert g.download().tobytes() == before.tobytes()   # queries never change the sketches
        g.ingest_pairs(pairs[:1000])                    # and ingest still works
        labels, ncc, _ = g.connected_components()
        assert np.array_equal(labels, restatement.exact_cc(V, np.concatenate([pairs, pairs[:1000]]))[1])
