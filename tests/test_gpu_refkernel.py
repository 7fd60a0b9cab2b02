"""The library against the reference's own GPU sketch-update kernel (src/cuda_kernel.cu:152-257 of the
reference), built for sm_100a from the reference sources into oracle/_ref by oracle/Makefile.

The reference kernel turns per-vertex batches (the GraphSketchDriver gutter form) into one delta sketch
per batch; the reference XORs those deltas into the vertex sketches on the host
(include/cuda_stream.h:171-182).  The XOR of all deltas must equal the library's device sketches byte
for byte.  The second test also times both on the same R-MAT records and prints one JSON line."""
import json

import numpy as np
import pytest

import gpusketch_b200 as gs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
bridge = pytest.importorskip("oracle.bridge")
if not bridge.ref_gpu_available():
    pytest.skip("oracle/_ref/libgsrefgpu.so not built (the reference tree was absent at build time)",
                allow_module_level=True)

THREADS, BATCHES_PER_LAUNCH = 1024, 540   # the reference's launch shape (include/cc_gpu_sketch_alg.h:14-33)


def run_reference(kernel, g, seed, pairs, deltas_for=None):
    """Runs the reference kernel over the stream in launches of 540 batches.  Returns the XOR of all
    deltas per source vertex for the vertices in deltas_for (all when None), as uint64 [V][nb][2], and
    the kernel time in ms (CUDA events around the launches only)."""
    geo = g.geometry
    nb = geo.num_buckets
    g_dict = {"num_samples": geo.num_samples, "num_buckets": nb, "num_columns": geo.num_columns,
              "bkt_per_col": geo.bkt_per_col}
    bs = int(g._lib.gs_desired_updates_per_batch(g._h))
    dsts, bsrc, bstart, bsize = bridge.ref_batches(pairs, bs)
    kernel.prepare(nb)
    d_dsts = torch.from_numpy(dsts.view(np.int32)).cuda()
    d_src = torch.from_numpy(bsrc.view(np.int32)).cuda()
    d_start = torch.from_numpy(bstart.view(np.int64)).cuda()
    d_size = torch.from_numpy(bsize.view(np.int64)).cuda()
    d_deltas = torch.empty((BATCHES_PER_LAUNCH, nb, 2), dtype=torch.int64, device="cuda")
    V = g.num_vertices
    want = np.ones(V, bool) if deltas_for is None else np.isin(np.arange(V), deltas_for)
    acc = np.zeros((V, nb, 2), np.uint64) if deltas_for is None else {int(v): np.zeros((nb, 2), np.uint64)
                                                                      for v in deltas_for}
    s = torch.cuda.current_stream()
    ms = 0.0
    for b0 in range(0, len(bsrc), BATCHES_PER_LAUNCH):
        n = min(BATCHES_PER_LAUNCH, len(bsrc) - b0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        kernel.sketch_update(THREADS, n, s.cuda_stream, d_dsts.data_ptr(), d_src.data_ptr() + 4 * b0,
                             d_size.data_ptr() + 8 * b0, d_start.data_ptr() + 8 * b0, g_dict, seed,
                             d_deltas.data_ptr())
        e1.record(s)
        sel = np.nonzero(want[bsrc[b0:b0 + n]])[0]
        if len(sel):
            rows = d_deltas[torch.from_numpy(sel).cuda()].cpu().numpy().view(np.uint64)
            for r, b in zip(rows, sel):
                acc[int(bsrc[b0 + b])] ^= r
        else:
            s.synchronize()
        ms += e0.elapsed_time(e1)
    return acc, ms, len(bsrc)


def test_sketches_equal_reference_kernel_deltas():
    V, seed = 1024, 0xC0FFEE
    pairs = gs.er_stream(V, 0.05, 0x5EED0001, 0.1, 0.5)
    kernel = bridge.RefGpuKernel()
    with gs.GraphSketch(V, seed) as g:
        g.ingest_pairs(pairs)
        ours = g.download().view(np.uint64).reshape(V, -1, 2)
        ref, _, _ = run_reference(kernel, g, seed, pairs)
    assert np.array_equal(ours, ref)


def test_rmat17_against_reference_kernel():
    """V = 2^17 R-MAT, 2^24 edge updates: the library's sketches equal the reference kernel's merged
    deltas on sampled vertices (hubs and leaves), and both are timed on the same records."""
    V, seed, n = 1 << 17, 0x5EED0002, 1 << 24
    d = torch.empty((n, 2), dtype=torch.int32, device="cuda")
    gs.rmat_stream(17, n, seed, out=d)
    pairs = d.cpu().numpy().view(np.uint32)
    kernel = bridge.RefGpuKernel()
    with gs.GraphSketch(V, 0xC0FFEE, max_batch_edges=n) as g:
        g.ingest_pairs(d)                      # warm-up, then cancelled by the second pass
        g.ingest_pairs(d)
        g.profile_enable(True)
        g.ingest_pairs(d)
        torch.cuda.synchronize()
        prof = g.profile_read()
        ours_ms = prof["ingest_ms"] + prof["bucket_ms"]
        deg = np.bincount(pairs.reshape(-1), minlength=V)
        sample = [int(np.argmax(deg)), 1, 2, 77, 4099, V - 1]
        ref, ref_ms, nbatches = run_reference(kernel, g, 0xC0FFEE, pairs, deltas_for=sample)
        for v in sample:
            mine = g.download(0, v, 1).view(np.uint64).reshape(-1, 2)
            assert np.array_equal(mine, ref[v]), v
    records = 2 * n
    print(json.dumps({"workload": "rmat17_2^24_edge_updates", "records": records, "reference_batches": nbatches,
                      "reference_kernel_ms": ref_ms, "reference_kernel_records_per_s": records / ref_ms * 1e3,
                      "library_bucket_plus_update_ms": ours_ms,
                      "library_records_per_s": records / ours_ms * 1e3,
                      "library_update_only_ms": prof["ingest_ms"],
                      "speedup_kernel_vs_kernel": ref_ms / ours_ms}))
