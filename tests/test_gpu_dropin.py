"""The C++ drop-in classes (gpusketch_b200/cpp) driven the way the reference's
tools/cuda_process_stream.cu drives CCGPUSketchAlg: binary stream file -> GraphSketchDriver ->
connected_components(), plus the write_binary checkpoint; the reference's own tool compiled unchanged
against those headers; and stream files read by the library itself (gs_ingest_stream_file)."""
import hashlib
import json
import os
import struct
import subprocess

import numpy as np
import pytest

import gpusketch_b200 as gs
from stream_file import REFERENCE_FIXTURE, read_stream_file, write_stream_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "gpusketch_b200", "_build", "cc_dropin_demo")
REF_TOOL = os.path.join(ROOT, "oracle", "_ref", "cuda_process_stream")
REF_MC_TOOL = os.path.join(ROOT, "oracle", "_ref", "min_cut")


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["file", "generic", "batches"])
def test_cpp_dropin_driver_matches_reference(tmp_path, golden_dir, mode):
    """The driver with the library reading the file, with reader threads pulling updates, and the
    reference's worker path (apply_update_batch from worker threads) all end at the reference's bytes."""
    assert os.path.exists(DEMO), "build() compiles the C++ drop-in demo"
    case = [c for c in json.load(open(os.path.join(golden_dir, "ref_digests.json"))) if c["name"] == "multiples_1024"][0]
    pairs = np.load(os.path.join(golden_dir, "multiples_1024_stream.npy"))
    stream = str(tmp_path / "multiples.data")
    ck = str(tmp_path / "ck.bin")
    write_stream_file(stream, 1024, pairs)
    queries = 1 if mode == "batches" else 3
    out = subprocess.run([DEMO, stream, str(int(case["seed"])), ck, str(queries), mode], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.startswith("num_cc=")]
    assert len(lines) == queries
    assert lines[-1].startswith("num_cc=78 ")
    data = open(ck, "rb").read()
    assert hashlib.sha256(data[20:]).hexdigest() == case["sketch_sha256"]


def test_stream_file_format_roundtrip(tmp_path):
    """The writer above produces the format the reference's fixture uses (9-byte records)."""
    pairs = np.array([[1, 2], [2, 1], [3, 4]], np.uint32)
    p = str(tmp_path / "s.data")
    write_stream_file(p, 8, pairs)
    d = open(p, "rb").read()
    assert len(d) == 12 + 9 * 3
    assert struct.unpack_from("<IQ", d, 0) == (8, 3)
    assert [d[12 + 9 * k] for k in range(3)] == [0, 1, 0]


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_TOOL), reason="the reference tool was not built (no reference tree)")
def test_reference_tool_builds_and_runs_unchanged_against_the_dropin():
    """tools/cuda_process_stream.cu of the reference, compiled without a single edit against
    gpusketch_b200/cpp (oracle/Makefile), processes the reference's own fixture: 78 components."""
    out = subprocess.run([REF_TOOL, REFERENCE_FIXTURE, "4", "2"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    cc = [l for l in out.stdout.splitlines() if l.startswith("Connected Components:")]
    assert len(cc) == 1 and int(cc[0].split(":")[1]) == 78, out.stdout


@pytest.mark.gpu
def test_stream_file_ingest_in_ranges(tmp_path, restatement):
    """gs_ingest_stream_file over several record ranges of a file spanning many staging slices equals
    the oracle fed the same records; the reference fixture gives its digest and 78 components."""
    import hashlib
    V, seed = 5000, 0x5EED3500
    rng = np.random.default_rng(35)
    pairs = rng.integers(0, V, size=(300_007, 2), dtype=np.uint32)
    path = str(tmp_path / "s.data")
    write_stream_file(path, V, pairs)
    with gs.GraphSketch(V, seed, max_batch_edges=1 << 13) as g:
        assert g.ingest_stream_file(path, 0, 100_000) == 100_000
        assert g.ingest_stream_file(path, 100_000, 77) == 77
        assert g.ingest_stream_file(path, 100_077) == len(pairs) - 100_077
        assert g.ingest_stream_file(path, len(pairs)) == 0
        sk = restatement.new_sketches(V)
        restatement.ingest(sk, V, seed, pairs)
        assert g.download().tobytes() == sk.tobytes()
    Vf, _, fpairs = read_stream_file(REFERENCE_FIXTURE)
    case = [c for c in json.load(open(os.path.join(os.path.dirname(REFERENCE_FIXTURE), "ref_digests.json")))
            if c["name"] == "multiples_file_1024"][0]
    with gs.GraphSketch(Vf, 0xC0FFEE) as g:
        assert g.ingest_stream_file(REFERENCE_FIXTURE) == len(fpairs)
        assert hashlib.sha256(g.download().tobytes()).hexdigest() == case["sketch_sha256"]
        assert g.connected_components()[1] == 78
    with gs.GraphSketch(100, 1) as g:
        with pytest.raises(gs.GpuSketchError) as e:
            g.ingest_stream_file(REFERENCE_FIXTURE)          # 1024 vertices in the file
        assert e.value.status == 1
        with pytest.raises(gs.GpuSketchError) as e:
            g.ingest_stream_file(str(tmp_path / "missing.data"))
        assert e.value.status == 7
    trunc = str(tmp_path / "t.data")
    open(trunc, "wb").write(open(path, "rb").read()[:12 + 9 * 1000 + 4])
    with gs.GraphSketch(V, seed) as g:
        with pytest.raises(gs.GpuSketchError) as e:
            g.ingest_stream_file(trunc)
        assert e.value.status == 7


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_MC_TOOL), reason="the reference tool was not built (no reference tree)")
@pytest.mark.parametrize("n_block,initial", [(512, 0), (8192, 1)])
def test_reference_min_cut_tool_runs_unchanged_against_the_dropin(tmp_path, n_block, initial):
    """tools/min_cut.cu of the reference, compiled without an edit against gpusketch_b200/cpp, on the
    planted-cut stream written as a binary stream file: at V=1024 its memory estimate allows no sketch
    graph, so every edge stays exact and the adjacency answers; at V=2^14 (the min-cut workload's size)
    one sketch level at its reduced_k factor (51 columns) certifies the cut with k=25 forests.  Both
    print the planted cut of 3."""
    from gpusketch_b200.workloads import planted_cut_stream
    recs, _ = planted_cut_stream(n_block)
    path = str(tmp_path / "planted.data")
    write_stream_file(path, 2 * n_block, recs)
    out = subprocess.run([REF_MC_TOOL, path, "4", "2", str(initial)], capture_output=True, text=True, timeout=900,
                         cwd=str(tmp_path))
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    final = [l for l in out.stdout.splitlines() if l.startswith("Final mincut value:")]
    assert len(final) == 1 and float(final[0].split(":")[1]) == 3.0, out.stdout[-3000:]
