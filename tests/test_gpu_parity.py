"""GPU parity: device sketches bit-identical to the oracle / the reference's own CCSketchAlg, and
connected components, forests and min cuts equal to exact answers.  All calls go through the C ABI."""
import hashlib
import json
import os

import numpy as np
import pytest

import gpusketch_b200 as gs
from stream_file import REFERENCE_FIXTURE, read_stream_file

pytestmark = pytest.mark.gpu

PLAIN_SEED = 0xC0FFEE


def sketch_bytes(g: gs.GraphSketch, level: int = 0) -> bytes:
    return g.download(level).tobytes()


def oracle_bytes(R, V, seed, pairs, factor=1.0) -> bytes:
    sk = R.new_sketches(V, factor)
    R.ingest(sk, V, seed, pairs, factor)
    return sk.tobytes()


def case_pairs(name, golden_dir):
    if name == "plain_cc_er1024":
        return gs.er_stream(1024, 0.05, 0x5EED0001, 0.10, 0.5)
    if name == "multiples_1024":
        return np.load(os.path.join(golden_dir, "multiples_1024_stream.npy"))
    if name == "er256_sparse":
        return gs.er_stream(256, 0.01, 11, 0.5, 0.2)
    if name == "er4096":
        return gs.er_stream(4096, 0.002, 13, 0.1, 0.5)
    if name == "multiples_file_1024":
        return read_stream_file(REFERENCE_FIXTURE)[2]
    if name == "rmat_v2p12":
        return gs.rmat_stream(12, 40000, 0x5EED0002)
    raise KeyError(name)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    return torch


def test_plain_cc_config(restatement, golden_dir):
    """ER G(1024, 0.05), 10% deleted, half re-inserted; sketch seed 0xC0FFEE; default params."""
    case = json.load(open(os.path.join(golden_dir, "ref_digests.json")))[0]
    pairs = case_pairs("plain_cc_er1024", golden_dir)
    with gs.GraphSketch(1024, PLAIN_SEED) as g:
        g.ingest_pairs(pairs)
        g.synchronize()
        b = sketch_bytes(g)
        assert hashlib.sha256(b).hexdigest() == case["sketch_sha256"]   # the reference's write_binary bytes
        assert b == oracle_bytes(restatement, 1024, PLAIN_SEED, pairs)
        labels, ncc, rounds = g.connected_components()
    exact_n, exact_labels = restatement.exact_cc(1024, pairs)
    assert ncc == exact_n == case["num_cc"]
    assert np.array_equal(labels, exact_labels)
    assert rounds == case["rounds"]


@pytest.mark.parametrize("device_input", [False, True])
def test_reference_digests(restatement, golden_dir, device_input, torch_cuda):
    for case in json.load(open(os.path.join(golden_dir, "ref_digests.json"))):
        pairs = case_pairs(case["name"], golden_dir)
        V, seed = case["V"], int(case["seed"])
        with gs.GraphSketch(V, seed) as g:
            if device_input:
                g.ingest_pairs(torch_cuda.from_numpy(pairs.astype(np.int32)).cuda())
            else:
                g.ingest_pairs(pairs)
            g.synchronize()
            assert hashlib.sha256(sketch_bytes(g)).hexdigest() == case["sketch_sha256"], case["name"]
            labels, ncc, rounds = g.connected_components()
        assert ncc == case["num_cc"] and rounds == case["rounds"], case["name"]
        _, exact = restatement.exact_cc(V, pairs)
        assert np.array_equal(labels, exact), case["name"]


@pytest.mark.parametrize("V,seed", [(2, 1), (3, 2**64 - 1), (17, 0), (256, 2**63), (1000, 12345),
                                    (4096, 0xDEADBEEFCAFEBABE), (16384, 77)])
def test_random_streams_bit_exact(restatement, V, seed):
    rng = np.random.default_rng(V * 7 + 1)
    n = min(60000, 30 * V)
    pairs = rng.integers(0, V, size=(n, 2), dtype=np.uint32)
    if V > 8:
        pairs = pairs[(pairs[:, 0] % 3) == (pairs[:, 1] % 3)]  # several components
    with gs.GraphSketch(V, seed) as g:
        g.ingest_pairs(pairs)
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, pairs)
        labels, ncc, rounds = g.connected_components()
    sk = restatement.new_sketches(V)
    restatement.ingest(sk, V, seed, pairs)
    st, olabels, orounds, _ = restatement.boruvka(sk, V, seed)
    assert st == 0 and np.array_equal(labels, olabels) and rounds == orounds
    assert ncc == restatement.exact_cc(V, pairs)[0]


def test_hub_vertex_spans_many_chunks(restatement):
    """A vertex with > 3 work chunks of records merges through the atomic path."""
    V, seed = 20000, 99
    star = np.stack([np.zeros(V - 1, np.uint32), np.arange(1, V, dtype=np.uint32)], 1)
    rng = np.random.default_rng(4)
    noise = rng.integers(0, V, size=(40000, 2), dtype=np.uint32)
    pairs = np.concatenate([star, noise, star[:5000]])          # 5000 star edges toggled off again
    with gs.GraphSketch(V, seed) as g:
        g.ingest_pairs(pairs)
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, pairs)
        labels, ncc, _ = g.connected_components()
    n, exact = restatement.exact_cc(V, pairs)
    assert ncc == n and np.array_equal(labels, exact)


@pytest.mark.parametrize("factor", [1.38, 1.45, 1.5, 1.6, 1.66, 1.75, 1.8, 1.9, 1.95, 2.0, 2.1, 2.2, 2.25, 2.3, 2.4])
def test_every_column_count_of_the_packed_layout(restatement, factor):
    """V=1024 with sketches_factor 1.38 .. 2.4 gives 19 .. 33 columns: spare lanes with and without an
    idle lane or a spare round without a column (19..23), every lane busy (24), no spare lanes
    (25..32), two columns per lane (33).  A hub vertex spans several work chunks."""
    V, seed = 1024, 0x5EED3000
    rng = np.random.default_rng(int(factor * 100))
    pairs = rng.integers(0, V, size=(20000, 2), dtype=np.uint32)
    hub = np.stack([np.full(3000, 7, np.uint32), rng.integers(0, V, 3000, dtype=np.uint32)], axis=1)
    pairs = np.concatenate([pairs, hub])
    with gs.GraphSketch(V, seed, sketches_factor=factor) as g:
        g.ingest_pairs(pairs)
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, pairs, factor), g.geometry.num_columns


@pytest.mark.parametrize("pinned", [False, True])
def test_host_input_across_many_staging_slices(restatement, pinned):
    """Host records larger than the staging ring move in slices through both pinned/device slots: pageable
    input is copied into the library's pinned ring, page-locked input is copied from in place.  The
    sketches equal the oracle's."""
    import torch
    V, seed = 4096, 0x5EED3100
    rng = np.random.default_rng(31)
    pairs = rng.integers(0, V, size=(200_003, 2), dtype=np.uint32)
    src = torch.from_numpy(pairs.view(np.int32)).pin_memory() if pinned else pairs
    with gs.GraphSketch(V, seed, max_batch_edges=1 << 14) as g:
        g.ingest_pairs(src)
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, pairs)
        labels, _, _ = g.connected_components()
    assert np.array_equal(labels, restatement.exact_cc(V, pairs)[1])


@pytest.mark.parametrize("on_device", [False, True])
def test_ingest_edges_src_dst_arrays(restatement, on_device):
    """gs_ingest_edges (separate src / dst arrays, interleaved on the device for device input, in several
    staging slices) gives the same sketches as the oracle."""
    import torch
    V, seed = 2048, 0x5EED3200
    rng = np.random.default_rng(32)
    pairs = rng.integers(0, V, size=(70_001, 2), dtype=np.uint32)
    src, dst = np.ascontiguousarray(pairs[:, 0]), np.ascontiguousarray(pairs[:, 1])
    if on_device:
        src, dst = torch.from_numpy(src.view(np.int32)).cuda(), torch.from_numpy(dst.view(np.int32)).cuda()
    with gs.GraphSketch(V, seed, max_batch_edges=1 << 14) as g:
        g.ingest_edges(src, dst)
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, pairs)


def test_device_views_produced_just_before_the_call(restatement):
    """Non-contiguous column views of records that a torch kernel has only just produced, on a side
    stream: the library orders its work after torch's current stream, and the contiguous temporaries
    stay valid until it has read them (a freed block is reused right after each call)."""
    import torch
    V, seed = 3000, 0x5EED3300
    side = torch.cuda.Stream()
    host = []
    with gs.GraphSketch(V, seed, max_batch_edges=1 << 13) as g:
        with torch.cuda.stream(side):
            gen = torch.Generator(device="cuda").manual_seed(77)
            for k in range(3):
                recs = torch.randint(0, V, (40_000, 3), device="cuda", dtype=torch.int32, generator=gen)
                if k % 2:
                    g.ingest_pairs(recs[:, 1:])               # a strided two-column view
                else:
                    g.ingest_edges(recs[:, 0], recs[:, 2])    # strided columns
                host.append(recs.cpu().numpy())
                del recs
                torch.full((1 << 22,), 7, dtype=torch.int32, device="cuda")  # takes freed blocks
            side.synchronize()
        got = sketch_bytes(g)
    pairs = np.concatenate([h[:, [1, 2]] if k % 2 else h[:, [0, 2]] for k, h in enumerate(host)]).astype(np.uint32)
    assert got == oracle_bytes(restatement, V, seed, pairs)


def test_more_than_32_columns(restatement):
    """sketches_factor 3 at V=4096 gives 49 columns: two columns per lane."""
    V, seed, f = 4096, 5, 3.0
    assert gs.geometry_for(V, f).num_columns > 32
    rng = np.random.default_rng(9)
    pairs = rng.integers(0, V, size=(50000, 2), dtype=np.uint32)
    with gs.GraphSketch(V, seed, sketches_factor=f) as g:
        g.ingest_pairs(pairs)
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, pairs, f)
        labels, _, _ = g.connected_components()
    assert np.array_equal(labels, restatement.exact_cc(V, pairs)[1])


def test_vertex_batches_apply_to_source_only(restatement):
    """apply_update_batch(src, dsts) XORs (src,dst) into src's sketch only, self-loops included."""
    V, seed = 512, 31
    rng = np.random.default_rng(6)
    srcs = rng.integers(0, V, 300).astype(np.uint32)
    sizes = rng.integers(0, 700, 300).astype(np.uint64)
    starts = np.zeros_like(sizes)
    np.cumsum(sizes[:-1], out=starts[1:])
    dsts = rng.integers(0, V, int(sizes.sum())).astype(np.uint32)
    dsts[:5] = srcs[0]
    with gs.GraphSketch(V, seed) as g:
        g.ingest_vertex_batches(srcs, starts, sizes, dsts)
        got = sketch_bytes(g)
    geo = restatement.geometry(V)
    nb = geo["num_buckets"]
    sk = restatement.new_sketches(V)
    for b in range(len(srcs)):
        s = int(srcs[b])
        one = sk[s * nb * 2:(s + 1) * nb * 2]
        for d in dsts[int(starts[b]):int(starts[b] + sizes[b])].tolist():
            e = (min(s, d) << 32) | max(s, d)
            restatement.sketch_update(one, V, seed, e)
    assert got == sk.tobytes()


@pytest.mark.parametrize("reg_depth", [0, 1])
def test_device_vertex_batches_past_the_owner_table(restatement, reg_depth):
    """Device-resident vertex batches are counted before the neighbour scratch grows to their size, so
    the chunk-owner table (sized by that scratch) covers only the first work chunks; the sketch update
    finds the vertex of every later chunk by search.  Small scratch, 32-record chunks: most chunks lie
    past the table.  The bytes equal the restatement's, for the packed and the one-column kernel."""
    import ctypes as C
    import torch
    from gpusketch_b200._native import check
    from gpusketch_b200.autotune import set_tuning
    V, seed = 512, 0x5EED0077
    rng = np.random.default_rng(77)
    srcs = rng.integers(0, V, 400).astype(np.uint32)
    sizes = rng.integers(0, 500, 400).astype(np.uint64)
    starts = np.zeros_like(sizes)
    np.cumsum(sizes[:-1], out=starts[1:])
    dsts = rng.integers(0, V, int(sizes.sum())).astype(np.uint32)
    with gs.GraphSketch(V, seed, max_batch_edges=1024) as g:
        set_tuning(g, 32, 8, reg_depth)
        d_srcs = torch.from_numpy(srcs.astype(np.int32)).cuda()
        d_starts = torch.from_numpy(starts.astype(np.int64)).cuda()
        d_sizes = torch.from_numpy(sizes.astype(np.int64)).cuda()
        d_dsts = torch.from_numpy(dsts.astype(np.int32)).cuda()
        torch.cuda.synchronize()
        check(g._lib.gs_ingest_vertex_batches(g._h, 0, d_srcs.data_ptr(), d_starts.data_ptr(), d_sizes.data_ptr(),
                                              len(srcs), d_dsts.data_ptr(), len(dsts), 1, None),
              "gs_ingest_vertex_batches")
        g.synchronize()
        got = sketch_bytes(g)
    nb = restatement.geometry(V)["num_buckets"]
    sk = restatement.new_sketches(V)
    for b in range(len(srcs)):
        s = int(srcs[b])
        one = sk[s * nb * 2:(s + 1) * nb * 2]
        for d in dsts[int(starts[b]):int(starts[b] + sizes[b])].tolist():
            restatement.sketch_update(one, V, seed, (min(s, d) << 32) | max(s, d))
    assert got == sk.tobytes()


def test_linearity_and_self_inverse(restatement):
    V, seed = 3000, 2024
    rng = np.random.default_rng(7)
    A = rng.integers(0, V, size=(30000, 2), dtype=np.uint32)
    B = rng.integers(0, V, size=(20000, 2), dtype=np.uint32)
    with gs.GraphSketch(V, seed) as g1, gs.GraphSketch(V, seed) as g2:
        g1.ingest_pairs(A); g1.ingest_pairs(B)
        g2.ingest_pairs(B); g2.ingest_pairs(np.concatenate([A[::-1]]))
        assert sketch_bytes(g1) == sketch_bytes(g2)
        g1.ingest_pairs(A); g1.ingest_pairs(B)
        assert not np.frombuffer(sketch_bytes(g1), np.uint64).any()   # merging the same delta twice gives ZERO


def test_edge_cases(restatement):
    V, seed = 100, 3
    with gs.GraphSketch(V, seed) as g:
        g.ingest_pairs(np.empty((0, 2), np.uint32))
        g.ingest_pairs(np.array([[5, 5], [7, 7]], np.uint32))      # self-loops cancel
        assert not np.frombuffer(sketch_bytes(g), np.uint64).any()
        labels, ncc, rounds = g.connected_components()
        assert ncc == V and rounds == 0                           # every sample is ZERO
        bad = np.array([[1, 2], [3, 100], [4, 5]], np.uint32)      # vertex 100 is out of range
        g.ingest_pairs(bad)
        with pytest.raises(gs.GpuSketchError) as e:
            g.synchronize()
        assert e.value.status == 1
        good = np.array([[1, 2], [4, 5]], np.uint32)
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, good)
        assert g.point_query(1, 2) and g.point_query(4, 5) and not g.point_query(1, 4)


def test_spanning_forest_and_disjoint_forests(restatement):
    V, seed = 2000, 8
    pairs = gs.er_stream(V, 0.004, 21, 0.2, 0.5)
    final = {tuple(e) for e in restatement.final_edges(V, pairs).tolist()}
    with gs.GraphSketch(V, seed) as g:
        g.ingest_pairs(pairs)
        before = sketch_bytes(g)
        f = g.spanning_forest()
        ncc_exact, exact = restatement.exact_cc(V, pairs)
        assert len(f) == V - ncc_exact and {tuple(e) for e in f.tolist()} <= final
        n2, lab2 = restatement.cc_of_edges(V, f)
        assert np.array_equal(lab2, exact)
        forests = g.disjoint_spanning_forests(3)
        assert sketch_bytes(g) == before                              # deletions were reverted
    remaining = set(final)
    for fo in forests:
        fe = {tuple(e) for e in fo.tolist()}
        assert fe <= remaining
        rem = np.asarray(sorted(remaining), np.uint32).reshape(-1, 2)
        n1, l1 = restatement.cc_of_edges(V, rem)
        n2, l2 = restatement.cc_of_edges(V, fo)
        assert np.array_equal(l1, l2) and len(fo) == V - n1
        remaining -= fe


def test_min_cut_levels_bit_exact(restatement):
    """Subgraph tagging: each edge goes to levels 0..min(tag, levels-1)."""
    V, seed, levels, L = 600, 17, 5, 19
    rng = np.random.default_rng(12)
    pairs = rng.integers(0, V, size=(20000, 2), dtype=np.uint32)
    with gs.GraphSketch(V, seed, num_levels=levels, num_subgraphs=L) as g:
        g.ingest_pairs(pairs)
        got = b"".join(sketch_bytes(g, lv) for lv in range(levels))
    sk = restatement.new_sketches(V, levels=levels)
    restatement.ingest_levels(sk, V, levels, L, seed, pairs)
    assert got == sk.tobytes()


def test_min_cut_planted_cut():
    """Two dense ER blocks joined by a planted cut of 3 edges: min cut 3 at level 0."""
    n, seed = 150, 0x5EED0003
    rng = np.random.default_rng(13)
    blocks = []
    for off in (0, n):
        a, b = np.triu_indices(n, 1)
        keep = rng.random(a.size) < 0.3
        blocks.append(np.stack([a[keep] + off, b[keep] + off], 1))
    cut = np.stack([rng.integers(0, n, 3), rng.integers(n, 2 * n, 3)], 1)
    pairs = np.concatenate(blocks + [cut]).astype(np.uint32)
    pairs = pairs[rng.permutation(len(pairs))]
    V = 2 * n
    L = 1 + 2 * int(np.log2(V))
    alg = gs.MCGPUSketchAlg(V, seed, num_subgraphs=L, max_sketch_graphs=4, k=4)
    alg.ingest_pairs(pairs)
    value, level, cut_at = alg.min_cut()
    assert (value, level, cut_at) == (3, 0, 3)


def test_checkpoint_roundtrip(restatement, tmp_path, golden_dir):
    case = json.load(open(os.path.join(golden_dir, "ref_digests.json")))[1]
    pairs = case_pairs("multiples_1024", golden_dir)
    path = str(tmp_path / "ck.bin")
    with gs.GraphSketch(1024, PLAIN_SEED) as g:
        g.ingest_pairs(pairs)
        g.write_binary(path)
    data = open(path, "rb").read()
    assert data[:20] == PLAIN_SEED.to_bytes(8, "little") + (1024).to_bytes(4, "little") + np.float64(1.0).tobytes()
    assert hashlib.sha256(data[20:]).hexdigest() == case["sketch_sha256"]
    g2 = gs.GraphSketch.read_binary(path)
    labels, ncc, _ = g2.connected_components()
    g2.close()
    assert ncc == 78


def test_reference_named_api(restatement, golden_dir):
    pairs = case_pairs("multiples_1024", golden_dir)
    alg = gs.CCGPUSketchAlg(1024, PLAIN_SEED, gs.CCAlgConfiguration().batch_factor(1), num_threads=4)
    # worker batches the way the driver delivers them: both directions, per source vertex
    src = np.concatenate([pairs[:, 0], pairs[:, 1]])
    dst = np.concatenate([pairs[:, 1], pairs[:, 0]])
    for v in np.unique(src):
        alg.apply_update_batch(int(v) % 4, int(v), dst[src == v])
    cc = alg.connected_components()
    assert cc.size() == 78
    ids = {frozenset(s) for s in cc.get_component_sets()}
    assert frozenset({2, 4, 6}) <= next(s for s in ids if 2 in s)
    # 3-6-2-10-5 joins 3 and 5; a prime p > 511 has no multiple below 1024 and stays alone
    assert alg.point_query(3, 9) and alg.point_query(3, 5) and not alg.point_query(3, 521)


def test_full_size_rmat_properties(restatement, torch_cuda):
    """V=2^17 R-MAT, 2^24 records generated on the device: exact partition, and per-vertex sketches
    of sampled vertices equal to their oracle sketch built from the vertex's own records."""
    torch = torch_cuda
    V, seed, n = 1 << 17, 0x5EED0002, 1 << 24
    d = torch.empty((n, 2), dtype=torch.int32, device="cuda")
    gs.rmat_stream(17, n, 0x5EED0002, out=d)
    host = d.cpu().numpy().astype(np.uint32)
    with gs.GraphSketch(V, seed) as g:
        g.ingest_pairs(d[: n // 2])
        g.ingest_pairs(d[n // 2:])
        labels, ncc, rounds = g.connected_components()
        sample = [0, 1, 2, 3, 1000, 65535, 131071]
        got = g.download()
    nexact, exact = restatement.exact_cc(V, host)
    assert ncc == nexact and np.array_equal(labels, exact)
    nb = restatement.geometry(V)["num_buckets"]
    for v in sample:
        mine = host[(host[:, 0] == v) | (host[:, 1] == v)]
        mine = mine[mine[:, 0] != mine[:, 1]]
        one = np.zeros(nb * 2, np.uint64)
        for a, b in mine.tolist():
            restatement.sketch_update(one, V, seed, (min(a, b) << 32) | max(a, b))
        assert got[v].tobytes() == one.tobytes(), v


def test_results_independent_of_tuning(restatement):
    """Every autotuner candidate produces the same bytes (XOR is order-independent)."""
    from gpusketch_b200.autotune import get_tuning, set_tuning
    V, seed = 5000, 41
    rng = np.random.default_rng(15)
    star = np.stack([np.zeros(3000, np.uint32), np.arange(1, 3001, dtype=np.uint32)], 1)
    pairs = np.concatenate([rng.integers(0, V, size=(60000, 2), dtype=np.uint32), star])
    want = oracle_bytes(restatement, V, seed, pairs)
    for chunk, warps, r in [(32, 1, 1), (1024, 4, 2), (4096, 8, 3), (100000, 16, 1), (777, 3, 2), (64, 2, 0),
                            (5000, 16, 0)]:
        with gs.GraphSketch(V, seed) as g:
            set_tuning(g, chunk, warps, r)
            assert get_tuning(g) == {"chunk": chunk, "warps_per_block": warps, "reg_depth": r}
            g.ingest_pairs(pairs)
            assert sketch_bytes(g) == want, (chunk, warps, r)


def test_autotune_keeps_sketches(torch_cuda):
    from gpusketch_b200.autotune import autotune
    V = 1 << 12
    d = torch_cuda.empty((1 << 18, 2), dtype=torch_cuda.int32, device="cuda")
    gs.rmat_stream(12, 1 << 18, 5, out=d)
    with gs.GraphSketch(V, 9) as g:
        g.ingest_pairs(d[:1000])
        before = sketch_bytes(g)
        best = autotune(g, d, chunks=(512, 4096), warps=(4, 8), reg_depths=(1, 2))
        assert sketch_bytes(g) == before
        assert best["reg_depth"] in (1, 2)


def test_min_cut_full_config():
    """V=2^14: two ER blocks of 8192 (p=0.3, ~20M edges) joined by 3 planted edges, 5% delete and
    re-insert, k=4 forests per level: the min cut is the planted 3 and its side is one block."""
    from gpusketch_b200.workloads import planted_cut_stream
    n = 8192
    recs, cross = planted_cut_stream(n)
    V = 2 * n
    L = 1 + 2 * int(np.log2(V))
    alg = gs.MCGPUSketchAlg(V, 0x5EED0003, num_subgraphs=L, max_sketch_graphs=4, k=4)
    alg.ingest_pairs(recs)
    value, level, cut_at, side = alg.sketches().min_cut(4)
    assert (value, level, cut_at) == (3, 0, 3)
    s = side.astype(bool)
    assert s[:n].all() != s[n:].all() and (s[:n].all() or not s[:n].any()) and (s[n:].all() or not s[n:].any())


def test_edge_store_tier_holds_the_deep_levels(restatement):
    """Edges whose subgraph tag passes the sketched levels are kept exactly (toggles flip them)."""
    V, seed, levels, L = 700, 23, 2, 19
    rng = np.random.default_rng(41)
    pairs = rng.integers(0, V, size=(40000, 2), dtype=np.uint32)
    pairs = np.concatenate([pairs, pairs[:5000]])            # some edges toggled back out
    with gs.GraphSketch(V, seed, num_levels=levels, num_subgraphs=L) as g:
        g.ingest_pairs(pairs[:20000])
        g.ingest_pairs(pairs[20000:])
        for t in (levels, levels + 2):
            got = g.edge_store_edges(t)
            final = restatement.final_edges(V, pairs)
            tags = np.array([(gs.hash64((int(a) << 32) | int(b), seed) | (1 << (L - 1))) for a, b in final.tolist()],
                            dtype=np.uint64)
            depth = np.array([(int(x) & -int(x)).bit_length() - 1 for x in tags])
            want = final[depth >= t]
            want = want[np.lexsort((want[:, 1], want[:, 0]))]
            assert np.array_equal(got, want), t
        g.clear()
        assert len(g.edge_store_edges()) == 0


def test_min_cut_falls_back_to_the_exact_tier():
    """One sketched level and a cut of 6 > k=4: level 0 certifies no cut below k, so the first
    unsketched level answers from the exact tier: the exact min cut of its edges, times 2."""
    n, seed = 120, 0x5EED0004
    rng = np.random.default_rng(14)
    blocks = []
    for off in (0, n):
        a, b = np.triu_indices(n, 1)
        keep = rng.random(a.size) < 0.5
        blocks.append(np.stack([a[keep] + off, b[keep] + off], 1))
    cross = np.stack([rng.integers(0, n, 6), rng.integers(n, 2 * n, 6)], 1)
    pairs = np.concatenate(blocks + [cross]).astype(np.uint32)
    V, L = 2 * n, 15
    with gs.GraphSketch(V, seed, num_levels=1, num_subgraphs=L) as g:
        g.ingest_pairs(pairs)
        value, level, cut_at, side = g.min_cut(4)
        assert level == 1 and value == cut_at * 2
        exact = g.edge_store_edges(1)
        lam, _ = gs.exact_min_cut(V, exact)
        assert cut_at == lam


@pytest.mark.parametrize("pinned", [True, False])
def test_async_ingest_and_query_overlap_phases(restatement, pinned):
    """gs_ingest_pairs_async + gs_connected_components_async: the next phase's records are queued
    (copies included) while the previous phase's query runs; every answer equals the exact partition of
    its own prefix, and the final sketches equal the oracle's, from page-locked and pageable input in
    several staging slices."""
    import torch
    V, seed, P = 6000, 0x5EED3400, 4
    rng = np.random.default_rng(34)
    pairs = rng.integers(0, V, size=(P * 70_001, 2), dtype=np.uint32)
    pairs = pairs[(pairs[:, 0] % 4) == (pairs[:, 1] % 4)]            # several components
    bounds = np.linspace(0, len(pairs), P + 1).astype(int)
    host = torch.from_numpy(pairs.view(np.int32)).pin_memory() if pinned else pairs
    with gs.GraphSketch(V, seed, max_batch_edges=1 << 14) as g:
        answers = []
        g.ingest_pairs_async(host[bounds[0]:bounds[1]])
        for p in range(P):
            g.connected_components_async()
            with pytest.raises(gs.GpuSketchError):
                g.connected_components_async()                   # one queued query at a time
            with pytest.raises(gs.GpuSketchError):
                g.connected_components()
            if p + 1 < P:
                g.ingest_pairs_async(host[bounds[p + 1]:bounds[p + 2]])   # queued behind the query
            answers.append(g.query_wait())
        for p, (labels, ncc, rounds) in enumerate(answers):
            n, exact = restatement.exact_cc(V, pairs[:bounds[p + 1]])
            assert ncc == n and np.array_equal(labels, exact), p
        g.synchronize()
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, pairs)
        # a later ingest makes the queued answer stale for point queries
        g.ingest_pairs(np.array([[1, 2]], np.uint32))
        want = restatement.exact_cc(V, np.concatenate([pairs, [[1, 2]]]).astype(np.uint32))[1]
        assert g.point_query(1, 2) == (want[1] == want[2]) == True
    with pytest.raises(gs.GpuSketchError):
        with gs.GraphSketch(V, seed) as g2:
            g2.query_wait()                                      # nothing queued


@pytest.mark.parametrize("V,n", [(5000, 60000), (1 << 17, 1 << 22)])
def test_complement_accumulation_equals_direct(restatement, V, n):
    """A sketch set that XORs to zero lets Boruvka take the largest component's merged column as the
    XOR of every vertex outside it.  The same sketches re-uploaded (after which the library no longer
    assumes that) run the direct accumulation: partitions, round counts and forests are equal, and
    equal the oracle's; both forests span it."""
    import torch
    d = torch.empty((n, 2), dtype=torch.int32, device="cuda")
    gs.rmat_stream(int(np.log2(V)) if V & (V - 1) == 0 else 13, n, 0x5EED3600, out=d)
    pairs = d.cpu().numpy().view(np.uint32) % np.uint32(V)
    with gs.GraphSketch(V, 0x5EED3601) as g:
        g.ingest_pairs(pairs)
        a_labels, a_ncc, a_rounds = g.connected_components()
        a_forest = g.spanning_forest()
        g.upload(g.download())                                   # same bytes, symmetry no longer assumed
        b_labels, b_ncc, b_rounds = g.connected_components()
        b_forest = g.spanning_forest()
    assert (a_ncc, a_rounds) == (b_ncc, b_rounds) and np.array_equal(a_labels, b_labels)
    # which edge of a cycle of sampled edges loses its union depends on timing: compare what forests are
    assert len(a_forest) == len(b_forest) == V - a_ncc
    for f in (a_forest, b_forest):
        assert np.array_equal(restatement.cc_of_edges(V, f)[1], a_labels)
    n_exact, exact = restatement.exact_cc(V, pairs)
    assert a_ncc == n_exact and np.array_equal(a_labels, exact)


def test_staging_ring_grows_with_the_host_input(restatement):
    """The page-locked ring starts small for small host batches and grows (after draining what is queued
    on it) when a larger batch arrives, also behind queued asynchronous work; gs_prepare_host_input sizes
    it up front.  The sketches equal the oracle's throughout."""
    import torch
    V, seed = 4000, 0x5EED3700
    rng = np.random.default_rng(37)
    small = rng.integers(0, V, size=(1000, 2), dtype=np.uint32)
    big = rng.integers(0, V, size=(3_000_001, 2), dtype=np.uint32)
    bigger = torch.from_numpy(rng.integers(0, V, size=(5_000_000, 2), dtype=np.uint32).view(np.int32)).pin_memory()
    with gs.GraphSketch(V, seed) as g:
        g.ingest_pairs(small)                       # a ring of 2^20 pairs
        g.ingest_pairs_async(big)                   # pageable: staged, grows the ring to 2^22
        g.ingest_pairs_async(bigger)                # page-locked and queued: grows again to 2^23
        g.synchronize()
        want = np.concatenate([small, big, bigger.numpy().view(np.uint32)])
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, want)
    with gs.GraphSketch(V, seed) as g:
        g.prepare_host_input(1 << 23)
        g.ingest_pairs(big)
        assert sketch_bytes(g) == oracle_bytes(restatement, V, seed, big)
