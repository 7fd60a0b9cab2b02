"""Parity pinned on the reference's own fixture and its own code at the headline sizes: the binary
stream file the reference's tests replay, the whole V=2^17 sketch set of the large-ingest stream
against the reference's CCSketchAlg, the benchmark's clear / ingest / query phase cycle phase by phase,
and the min-cut subgraph fan-out against the reference's MCSketchAlg.  Everything goes through the C
ABI; every comparison is bit-exact (integer work, tolerance 0)."""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import gpusketch_b200 as gs
from oracle import RefCC, RefMC, ref_available
from stream_file import REFERENCE_FIXTURE, read_stream_file

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "gpusketch_b200", "_build", "cc_dropin_demo")
SEED = 0xC0FFEE


def _digest(golden_dir, name):
    return [c for c in json.load(open(os.path.join(golden_dir, "ref_digests.json"))) if c["name"] == name][0]


def _label_checksum(labels) -> int:
    s = 0
    for x in labels.tolist():
        s = (s * 1000003 + x) & (2**64 - 1)
    return s


def test_reference_fixture_file_through_the_c_abi(restatement, golden_dir):
    """test/cc_alg_test.cpp:300-350 (MTStreamWithMultipleQueries) on the library: the reference's binary
    fixture replayed in file order with a query after every n/10 records; every partition equals the
    exact partition of the prefix, the final one has 78 components, and the final sketch bytes equal
    the reference CCSketchAlg's."""
    V, _, pairs = read_stream_file(REFERENCE_FIXTURE)
    case = _digest(golden_dir, "multiples_file_1024")
    per = len(pairs) // 10
    with gs.GraphSketch(V, SEED) as g:
        done = 0
        for q in range(1, 11):
            upto = per * q if q < 10 else len(pairs)
            g.ingest_pairs(pairs[done:upto])
            done = upto
            labels, ncc, _ = g.connected_components()
            n, exact = restatement.exact_cc(V, pairs[:upto])
            assert ncc == n and np.array_equal(labels, exact), q
        assert ncc == 78
        assert hashlib.sha256(g.download().tobytes()).hexdigest() == case["sketch_sha256"]


def test_reference_fixture_file_through_the_cpp_driver(tmp_path, restatement, golden_dir):
    """The same file read by the C++ BinaryFileStream and driven through GraphSketchDriver ->
    CCGPUSketchAlg with the reference test's ten query points; the write_binary checkpoint equals the
    reference's bytes."""
    assert os.path.exists(DEMO), "build() compiles the C++ drop-in demo"
    V, _, pairs = read_stream_file(REFERENCE_FIXTURE)
    case = _digest(golden_dir, "multiples_file_1024")
    ck = str(tmp_path / "ck.bin")
    out = subprocess.run([DEMO, REFERENCE_FIXTURE, str(SEED), ck, "10"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.startswith("num_cc=")]
    assert len(lines) == 10
    per = len(pairs) // 10
    for q, line in enumerate(lines, 1):
        upto = per * q if q < 10 else len(pairs)
        n, exact = restatement.exact_cc(V, pairs[:upto])
        fields = dict(kv.split("=") for kv in line.split())
        assert int(fields["num_cc"]) == n and int(fields["label_checksum"], 16) == _label_checksum(exact), q
    assert lines[-1].startswith("num_cc=78 ")
    data = open(ck, "rb").read()
    assert hashlib.sha256(data[20:]).hexdigest() == case["sketch_sha256"]


def test_whole_v2p17_sketch_set_equals_reference():
    """V=2^17, 2^25 records of the benchmark's R-MAT stream generated on the device and ingested in two
    device-resident calls: all 131072 x 817 buckets (1.7 GB) equal the reference CCSketchAlg's
    sketches after the same records go through its apply_update_batch, and the partition and round
    count equal its connected_components()."""
    import torch
    V, n = 1 << 17, 1 << 25
    d = torch.empty((n, 2), dtype=torch.int32, device="cuda")
    gs.rmat_stream(17, n, 0x5EED0002, out=d)
    host = d.cpu().numpy().view(np.uint32)
    with gs.GraphSketch(V, SEED) as g:
        g.ingest_pairs(d[: n // 2])
        g.ingest_pairs(d[n // 2:])
        labels, ncc, rounds = g.connected_components()
        got = g.download().view(np.uint64).reshape(V, -1)
    del d
    ref = RefCC(V, SEED, 1.0, workers=len(os.sched_getaffinity(0)))
    ref.ingest(host)
    want = ref.sketch_array(got.shape[1] // 2)
    diff = np.flatnonzero((got != want).any(axis=1))
    assert diff.size == 0, f"{diff.size} vertex sketches differ, first {diff[:8].tolist()}"
    rlabels, rncc, rrounds = ref.connected_components()
    ref.close()
    assert ncc == rncc and rounds == rrounds and np.array_equal(labels, rlabels)


def test_benchmark_phase_cycle_phase_by_phase(restatement):
    """The benchmark's step structure at a reduced size: twice (clear, then 4 x (ingest a 2^22-record
    slice of the R-MAT stream + connected_components())) at V=2^17.  Every phase's partition and round
    count equal the reference CCSketchAlg fed the same slices (and its partition the exact one)."""
    import torch
    V, phase, P = 1 << 17, 1 << 22, 4
    d = torch.empty((P * phase, 2), dtype=torch.int32, device="cuda")
    gs.rmat_stream(17, P * phase, 0x5EED0002, out=d)
    host = d.cpu().numpy().view(np.uint32)
    T = len(os.sched_getaffinity(0))
    expect = []
    ref = RefCC(V, SEED, 1.0, workers=T)
    for p in range(P):
        ref.ingest(host[p * phase:(p + 1) * phase])
        labels, ncc, rounds = ref.connected_components()
        expect.append((labels, ncc, rounds))
    ref.close()
    _, exact = restatement.exact_cc(V, host)
    assert np.array_equal(expect[-1][0], exact)
    with gs.GraphSketch(V, SEED, max_batch_edges=phase) as g:
        for step in range(2):
            g.clear()
            for p in range(P):
                g.ingest_pairs(d[p * phase:(p + 1) * phase])
                labels, ncc, rounds = g.connected_components()
                el, encc, erounds = expect[p]
                assert (ncc, rounds) == (encc, erounds) and np.array_equal(labels, el), (step, p)


def test_min_cut_levels_equal_reference_mcsketchalg(restatement):
    """Subgraph tagging on the device against the reference's own MCSketchAlg fed through its GPU
    driver's fan-out (tag get_index_depth(e, seed, L-1), levels 0..min(tag, levels-1),
    src/mc_gpu_sketch_alg.cpp:139-178): every level's sketch bytes are equal."""
    for V, seed, levels, L, n in [(600, 17, 5, 19, 20000), (2048, 0x5EED0003, 4, 23, 200000)]:
        rng = np.random.default_rng(V + levels)
        pairs = rng.integers(0, V, size=(n, 2), dtype=np.uint32)
        ref = RefMC(V, seed, levels)
        ref.ingest_tagged(pairs, L)
        nb = gs.geometry_for(V).num_buckets
        with gs.GraphSketch(V, seed, num_levels=levels, num_subgraphs=L) as g:
            g.ingest_pairs(pairs[: n // 3])
            g.ingest_pairs(pairs[n // 3:])
            for lv in range(levels):
                assert g.download(lv).tobytes() == ref.level_bytes(lv, nb), (V, lv)
        ref.close()
