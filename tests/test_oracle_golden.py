"""The oracle restatement pinned against golden vectors and against the reference's own sources."""
import json
import os

import numpy as np
import pytest

from oracle import Restatement, ref_available
from stream_file import REFERENCE_FIXTURE, read_stream_file


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
        elif case["name"] == "multiples_file_1024":
            pairs = read_stream_file(REFERENCE_FIXTURE)[2]
        elif case["name"] == "rmat_v2p12":
            pairs = gs.rmat_stream(12, 40000, 0x5EED0002)
        else:
            raise KeyError(case["name"])
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


def test_reference_stream_fixture(restatement, golden_dir):
    """The reference's own binary fixture (test/res/multiples_graph_1024_stream.data, copied verbatim):
    8528 records of which 1661 deletes, each delete toggling a present edge, ending at the multiples
    graph of test/res/multiples_graph_1024.txt (78 components, test/cc_alg_test.cpp:300-350).  The
    restatement's sketch bytes equal the reference digest, and at each of the reference test's ten query
    points its Boruvka partition equals the exact partition of the prefix."""
    import hashlib
    V, types, pairs = read_stream_file(REFERENCE_FIXTURE)
    assert (V, len(pairs), int((types == 1).sum())) == (1024, 8528, 1661)
    present = set()
    for t, (a, b) in zip(types.tolist(), pairs.tolist()):
        e = (min(a, b), max(a, b))
        assert (t == 1) == (e in present)
        present.symmetric_difference_update({e})
    rule = {(i, j) for i in range(2, 1024) for j in range(2 * i, 1024, i)}
    assert present == rule
    case = [c for c in json.load(open(os.path.join(golden_dir, "ref_digests.json")))
            if c["name"] == "multiples_file_1024"][0]
    sk = restatement.new_sketches(V)
    restatement.ingest(sk, V, 0xC0FFEE, pairs)
    assert hashlib.sha256(sk.tobytes()).hexdigest() == case["sketch_sha256"]
    per = len(pairs) // 10
    for q in range(1, 11):
        upto = per * q if q < 10 else len(pairs)
        sk = restatement.new_sketches(V)
        restatement.ingest(sk, V, 0xC0FFEE, pairs[:upto])
        st, labels, _, _ = restatement.boruvka(sk, V, 0xC0FFEE)
        n, exact = restatement.exact_cc(V, pairs[:upto])
        assert st == 0 and np.array_equal(labels, exact), q
    assert n == 78


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_reference_fixture_through_reference_batches(restatement, golden_dir):
    """The reference's CCSketchAlg fed the fixture's records the way its driver does (both directions,
    per source vertex, through apply_update_batch) gives the digest's bytes."""
    import hashlib
    from oracle import RefCC
    V, _, pairs = read_stream_file(REFERENCE_FIXTURE)
    case = [c for c in json.load(open(os.path.join(golden_dir, "ref_digests.json")))
            if c["name"] == "multiples_file_1024"][0]
    ref = RefCC(V, 0xC0FFEE, 1.0, workers=4)
    ref.ingest(pairs, threads=4)
    assert hashlib.sha256(ref.sketch_bytes()).hexdigest() == case["sketch_sha256"]
    labels, ncc, rounds = ref.connected_components()
    assert (ncc, rounds) == (case["num_cc"], case["rounds"]) == (78, 6)
    ref.close()


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_min_cut_level_fanout_equals_reference(restatement):
    """The restatement's subgraph tagging (levels 0..min(tag, levels-1), tag = get_index_depth(e, seed,
    L-1)) equals the reference MCSketchAlg fed through the reference GPU driver's fan-out
    (src/mc_gpu_sketch_alg.cpp:139-178) level by level."""
    from oracle import RefMC
    for V, seed, levels, L, n in [(600, 17, 5, 19, 20000), (1000, 2**63 + 11, 3, 21, 30000)]:
        rng = np.random.default_rng(V)
        pairs = rng.integers(0, V, size=(n, 2), dtype=np.uint32)
        ref = RefMC(V, seed, levels)
        ref.ingest_tagged(pairs, L)
        nb = restatement.geometry(V)["num_buckets"]
        sk = restatement.new_sketches(V, levels=levels)
        restatement.ingest_levels(sk, V, levels, L, seed, pairs)
        for g in range(levels):
            assert ref.level_bytes(g, nb) == sk[g * V * nb * 2:(g + 1) * V * nb * 2].tobytes(), (V, g)
        ref.close()
