"""The oracle restatement pinned against golden vectors and against the reference's own sources."""
import json
import os

import numpy as np
import pytest

from oracle import Restatement, ref_available


def test_xxh3_golden_vectors(restatement, golden_dir):
    vecs = json.load(open(os.path.join(golden_dir, "xxh3_vectors.json")))
    assert len(vecs) > 300
    for k, s, h in vecs:
        assert restatement.xxh3(int(k), int(s)) == int(h), (k, s)


def test_geometry_matches_reference_table(restatement, golden_dir):
    for V, f, nb in json.load(open(os.path.join(golden_dir, "geometry.json"))):
        assert restatement.geometry(V, f)["num_buckets"] == nb, (V, f)


def test_geometry_known_sizes(restatement):
    # include/sketch.h sizing at the benchmark sizes
    assert restatement.geometry(1024)["num_buckets"] == 361
    g = restatement.geometry(131072)
    assert (g["num_columns"], g["bkt_per_col"], g["num_buckets"]) == (24, 34, 817)
    assert restatement.geometry(65536)["bkt_per_col"] == 33  # 32 is bumped off a multiple of 16


def test_depth_is_ctz_of_column_hash(restatement):
    rng = np.random.default_rng(3)
    for _ in range(200):
        e = int(rng.integers(0, 2**62)); s = int(rng.integers(0, 2**62)); md = int(rng.integers(1, 40))
        h = restatement.xxh3(e, s) | (1 << md)
        assert restatement.depth(e, s, md) == (h & -h).bit_length() - 1


def test_multiples_graph_known_answer(restatement, golden_dir):
    """test/cc_alg_test.cpp:41-57: the multiples graph has 78 components."""
    pairs = np.load(os.path.join(golden_dir, "multiples_1024_stream.npy"))
    assert pairs.shape == (8528, 2)
    ncc, _ = restatement.exact_cc(1024, pairs)
    assert ncc == 78
    sk = restatement.new_sketches(1024)
    restatement.ingest(sk, 1024, 0xC0FFEE, pairs)
    st, labels, rounds, forest = restatement.boruvka(sk, 1024, 0xC0FFEE)
    assert st == 0 and len(set(labels.tolist())) == 78
    assert len(forest) == 1024 - 78


def test_sketch_digests_match_reference(restatement, golden_dir):
    """Oracle sketches reproduce the reference CCSketchAlg's write_binary bytes (golden sha256)."""
    import hashlib
    import gpusketch_b200 as gs
    for case in json.load(open(os.path.join(golden_dir, "ref_digests.json"))):
        V, seed = case["V"], int(case["seed"])
        if case["name"] == "plain_cc_er1024":
            pairs = gs.er_stream(1024, 0.05, 0x5EED0001, 0.10, 0.5)
        elif case["name"] == "multiples_1024":
            pairs = np.load(os.path.join(golden_dir, "multiples_1024_stream.npy"))
        elif case["name"] == "er256_sparse":
            pairs = gs.er_stream(256, 0.01, 11, 0.5, 0.2)
        elif case["name"] == "er4096":
            pairs = gs.er_stream(4096, 0.002, 13, 0.1, 0.5)
        else:
            pairs = gs.rmat_stream(12, 40000, 0x5EED0002)
        assert hashlib.sha256(np.ascontiguousarray(pairs, np.uint32).tobytes()).hexdigest() == case["pairs_sha256"]
        sk = restatement.new_sketches(V)
        restatement.ingest(sk, V, seed, pairs)
        assert hashlib.sha256(sk.tobytes()).hexdigest() == case["sketch_sha256"], case["name"]
        st, labels, rounds, _ = restatement.boruvka(sk, V, seed)
        assert st == 0 and len(set(labels.tolist())) == case["num_cc"] and rounds == case["rounds"], case["name"]


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_restatement_equals_reference_build(restatement):
    """Sketch bytes, partition and round count of the restatement equal the compiled reference's."""
    from oracle import RefCC
    rng = np.random.default_rng(11)
    for V, seed, n in [(300, 99, 3000), (1024, 2**64 - 3, 12000), (2000, 0xABCDEF, 9000)]:
        pairs = rng.integers(0, V, size=(n, 2), dtype=np.uint32)
        pairs = pairs[(pairs[:, 0] % 5) == (pairs[:, 1] % 5)]   # several components
        ref = RefCC(V, seed, 1.0, workers=3)
        ref.ingest(pairs, threads=3)
        sk = restatement.new_sketches(V)
        restatement.ingest(sk, V, seed, pairs)
        assert ref.sketch_bytes() == sk.tobytes()
        labels, ncc, rounds = ref.connected_components()
        st, ol, orounds, _ = restatement.boruvka(sk, V, seed)
        assert st == 0 and np.array_equal(labels, ol) and rounds == orounds
        exact, el = restatement.exact_cc(V, pairs)
        assert np.array_equal(el, ol) and exact == ncc
        ref.close()


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_restatement_k_forests_are_disjoint_spanning_forests(restatement):
    """MCSketchAlg::calc_disjoint_spanning_forests semantics: edge-disjoint, each a spanning forest of
    what remains (test/util/graph_verifier.cpp:107-149)."""
    from oracle import RefMC
    V, seed, k = 200, 77, 3
    rng = np.random.default_rng(5)
    pairs = rng.integers(0, V, size=(3000, 2), dtype=np.uint32)
    final = restatement.final_edges(V, pairs)
    sk = restatement.new_sketches(V)
    restatement.ingest(sk, V, seed, pairs)
    before = sk.copy()
    st, forests = restatement.k_forests(sk, V, seed, k)
    assert st == 0 and np.array_equal(sk, before)  # restored
    remaining = {tuple(e) for e in final.tolist()}
    for f in forests:
        fe = {tuple(e) for e in f.tolist()}
        assert fe <= remaining
        n1, l1 = restatement.cc_of_edges(V, np.asarray(sorted(remaining), np.uint32))
        n2, l2 = restatement.cc_of_edges(V, f)
        assert np.array_equal(l1, l2) and len(f) == V - n1
        remaining -= fe
    ref = RefMC(V, seed, 1)
    for a, b in pairs.tolist():
        ref.update(0, a, b)
    rc, rforests = ref.k_forests(0, k)
    assert rc == 0 and [len(f) for f in rforests] == [len(f) for f in forests]
