"""Eager DSU: connectivity answered without Boruvka while the stream has only grown it, and exact
answers (tolerance 0) whether a query is served from the DSU or by Boruvka."""
import numpy as np
import pytest

import gpusketch_b200 as gs

pytestmark = pytest.mark.gpu


def exact_labels(restatement, V, pairs):
    _, lab = restatement.exact_cc(V, np.asarray(pairs, np.uint32).reshape(-1, 2))
    return lab


def test_insert_only_batches_never_run_boruvka(restatement):
    V = 2000
    recs = gs.er_stream(V, 0.002, 61)            # inserts only
    with gs.GraphSketch(V, 7) as g:
        g.set_eager_dsu(True)
        assert g.has_cached_query()              # the empty graph
        g.profile_enable(True)
        cuts = np.linspace(0, len(recs), 6).astype(int)
        for i in range(5):
            g.ingest_pairs(recs[cuts[i]:cuts[i + 1]])
            assert g.has_cached_query()
            labels, ncc, rounds = g.connected_components()
            assert rounds == 0
            assert np.array_equal(labels, exact_labels(restatement, V, recs[:cuts[i + 1]]))
        assert g.profile_read()["query_launches"] == 0
        with gs.GraphSketch(V, 7) as plain:      # the sketches are the same with or without it
            plain.ingest_pairs(recs)
            assert plain.download().tobytes() == g.download().tobytes()


def test_forest_edge_delete_invalidates_and_boruvka_restores(restatement):
    V = 64
    path = np.array([[0, 1], [1, 2], [2, 3]], np.uint32)
    with gs.GraphSketch(V, 11) as g:
        g.set_eager_dsu(True)
        g.ingest_pairs(path)
        assert g.has_cached_query()
        labels, ncc, _ = g.connected_components()
        assert ncc == V - 3 and labels[3] == 0
        g.ingest_pairs(np.array([[2, 1]], np.uint32))      # toggles forest edge {1,2}: a delete
        assert not g.has_cached_query()
        labels, ncc, rounds = g.connected_components()      # Boruvka
        assert rounds > 0 and ncc == V - 2 and labels[1] == 0 and labels[2] == 2 and labels[3] == 2
        assert g.has_cached_query()                          # rebuilt from Boruvka's forest
        g.ingest_pairs(np.array([[1, 2]], np.uint32))       # inserted again: merges
        assert g.has_cached_query()
        labels, ncc, rounds = g.connected_components()
        assert rounds == 0 and ncc == V - 3 and labels[3] == 0


def test_edge_toggled_twice_in_one_batch(restatement):
    """Insert then delete of one edge in the same batch: the eager pass may not keep it connected."""
    V = 32
    batch = np.array([[0, 1], [1, 2], [2, 1]], np.uint32)
    with gs.GraphSketch(V, 13) as g:
        g.set_eager_dsu(True)
        g.ingest_pairs(batch)
        assert not g.has_cached_query()
        labels, _, _ = g.connected_components()
        assert np.array_equal(labels, exact_labels(restatement, V, batch))
        assert labels[2] == 2 and labels[1] == 0


def test_random_streams_exact_cached_or_not(restatement):
    rng = np.random.default_rng(62)
    for V, p, seed in [(500, 0.01, 1), (3000, 0.001, 2), (1 << 13, 0.0004, 3)]:
        recs = gs.er_stream(V, p, seed, 0.2, 0.5)
        cached = 0
        with gs.GraphSketch(V, seed) as g:
            g.set_eager_dsu(True)
            pos = 0
            while pos < len(recs):
                step = int(rng.integers(1, max(2, len(recs) // 8)))
                g.ingest_pairs(recs[pos:pos + step])
                pos += step
                cached += g.has_cached_query()
                labels, _, _ = g.connected_components()
                assert np.array_equal(labels, exact_labels(restatement, V, recs[:pos])), (V, pos)
        assert cached > 0


def test_spanning_forest_from_the_eager_dsu(restatement):
    V = 1500
    recs = gs.er_stream(V, 0.002, 63)
    with gs.GraphSketch(V, 5) as g:
        g.set_eager_dsu(True)
        g.ingest_pairs(recs)
        assert g.has_cached_query()
        forest = g.spanning_forest()
        labels, ncc, rounds = g.connected_components()
        assert rounds == 0 and len(forest) == V - ncc
        present = {(min(a, b), max(a, b)) for a, b in restatement.final_edges(V, recs).tolist()}
        assert all((int(a), int(b)) in present for a, b in forest)
        assert np.array_equal(exact_labels(restatement, V, forest), labels)


def test_clear_upload_and_vertex_batches():
    V = 256
    recs = gs.er_stream(V, 0.02, 64)
    with gs.GraphSketch(V, 9) as g:
        g.ingest_pairs(recs)
        g.set_eager_dsu(True)                    # enabled on a non-empty graph: first query rebuilds
        assert not g.has_cached_query()
        g.connected_components()
        assert g.has_cached_query()
        g.clear()
        assert g.has_cached_query()
        labels, ncc, _ = g.connected_components()
        assert ncc == V and np.array_equal(labels, np.arange(V))
        g.ingest_vertex_batches([1], [0], [1], [2])   # one-sided update: the DSU cannot follow it
        assert not g.has_cached_query()


def test_min_cut_graphs_reject_the_eager_dsu():
    with gs.GraphSketch(128, 3, num_levels=3) as g:
        with pytest.raises(gs.GpuSketchError):
            g.set_eager_dsu(True)
