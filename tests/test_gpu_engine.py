"""Multi-tenant engine: each tenant's sketches and answers equal the same graph run alone.

Tenants of uneven sizes, seeds and sketch factors share one arena and one ingest call whose slices
interleave them; every tenant's sketch bytes must equal a solo GraphSketch (and the oracle), and
its connected components must equal the solo query and the exact partition (XOR linearity: the
tolerance is zero).  Admission, removal and slot reuse are checked against the byte accounting.
"""
import os

import numpy as np
import pytest

import gpusketch_b200 as gs
from gpusketch_b200 import _native
from gpusketch_b200.engine import SketchEngine, tenant_bytes

pytestmark = pytest.mark.gpu

TENANTS = [  # (V, seed, sketches_factor, stream)
    (300, 0x5EED1000, 1.0, lambda: gs.er_stream(300, 0.05, 1, 0.1, 0.5)),
    (1024, 0x5EED1001, 1.0, lambda: gs.er_stream(1024, 0.01, 2, 0.1, 0.5)),
    (4096, 0x5EED1002, 1.0, lambda: gs.rmat_stream(12, 30000, 3)),
    (777, 0x5EED1003, 1.5, lambda: gs.er_stream(777, 0.004, 4, 0.1, 0.5)),
    (2000, 0x5EED1004, 0.5, lambda: gs.er_stream(2000, 0.0015, 5, 0.3, 0.3)),
]


def interleaved_slices(streams, pieces, rng):
    """One ingest call's tables: every stream cut into `pieces` runs, runs shuffled across tenants."""
    runs = []
    for t, a in streams:
        cuts = np.linspace(0, len(a), pieces + 1).astype(int)
        runs += [(t, a[cuts[i]:cuts[i + 1]]) for i in range(pieces)]
    order = rng.permutation(len(runs))
    tens, offs, parts = [], [0], []
    for i in order:
        t, a = runs[i]
        tens.append(t)
        parts.append(a)
        offs.append(offs[-1] + len(a))
    return np.array(tens, np.uint32), np.array(offs, np.uint64), np.concatenate(parts)


def solo(V, seed, factor, pairs):
    with gs.GraphSketch(V, seed, sketches_factor=factor) as g:
        g.ingest_pairs(pairs)
        labels, ncc, rounds = g.connected_components()
        return g.download().tobytes(), labels, ncc, rounds


def make_engine(budget_mb=256, max_tenants=16, max_vertices=1 << 16, max_tenant_vertices=1 << 14):
    return SketchEngine(budget_mb << 20, max_tenants, max_vertices, max_tenant_vertices, max_batch_edges=1 << 20)


@pytest.mark.parametrize("device_input", [False, True])
def test_tenants_match_solo_runs(restatement, device_input):
    import torch
    rng = np.random.default_rng(7)
    with make_engine() as e:
        ids, streams = [], []
        for V, seed, f, gen in TENANTS:
            t = e.add_tenant(V, seed, f)
            ids.append(t)
            streams.append((t, gen()))
        tens, offs, pairs = interleaved_slices(streams, 3, rng)
        if device_input:
            e.ingest(tens, offs, torch.from_numpy(pairs.astype(np.int32)).cuda())
        else:
            e.ingest(tens, offs, pairs)
        e.synchronize()
        res = e.connected_components(ids)
        for (V, seed, f, _), (t, a) in zip(TENANTS, streams):
            sk, labels, ncc, rounds = solo(V, seed, f, a)
            assert e.download(t).tobytes() == sk, t
            r = res[t]
            assert (r.num_cc, r.rounds) == (ncc, rounds), t
            assert np.array_equal(r.labels, labels), t
            _, exact = restatement.exact_cc(V, a)
            assert np.array_equal(r.labels, exact), t
        # the smallest tenants against the oracle restatement as well
        for (V, seed, f, _), (t, a) in list(zip(TENANTS, streams))[:2]:
            sk = restatement.new_sketches(V, f)
            restatement.ingest(sk, V, seed, a, f)
            assert e.download(t).tobytes() == sk.tobytes()


def test_tiny_and_large_tenants_share_a_launch(restatement):
    """Tenants of at most 23 vertices have fewer buckets per column (bkt_per_col < 10) than the sketch
    update keeps shared-memory rows, so their deepest buckets are below the rows' end while a large
    tenant's go past it to HBM.  One launch updates both kinds: every tenant's bytes equal a solo run
    and the oracle."""
    rng = np.random.default_rng(21)
    specs = [
        (3, 0x5EED2000, 1.0, lambda: gs.er_stream(3, 0.9, 21, 0.1, 0.5)),
        (12, 0x5EED2001, 1.0, lambda: gs.er_stream(12, 0.5, 22, 0.1, 0.5)),
        (23, 0x5EED2002, 1.0, lambda: gs.er_stream(23, 0.3, 23, 0.1, 0.5)),
        (4096, 0x5EED2003, 1.0, lambda: gs.rmat_stream(12, 60000, 24)),
        (300, 0x5EED2004, 1.0, lambda: gs.er_stream(300, 0.05, 25, 0.1, 0.5)),
    ]
    assert gs.geometry_for(12).bkt_per_col < 10 <= gs.geometry_for(4096).bkt_per_col
    with make_engine() as e:
        ids, streams = [], []
        for V, seed, f, gen in specs:
            t = e.add_tenant(V, seed, f)
            ids.append(t)
            streams.append((t, gen()))
        tens, offs, pairs = interleaved_slices(streams, 3, rng)
        e.ingest(tens, offs, pairs)
        res = e.connected_components(ids)
        for (V, seed, f, _), (t, a) in zip(specs, streams):
            sk, labels, ncc, rounds = solo(V, seed, f, a)
            assert e.download(t).tobytes() == sk, t
            assert np.array_equal(res[t].labels, labels), t
            ref = restatement.new_sketches(V, f)
            restatement.ingest(ref, V, seed, a, f)
            assert e.download(t).tobytes() == ref.tobytes(), t


def test_large_vertex_space_two_word_records(restatement):
    """In a 2^22-id vertex space a bucket-local key (11 bits) and a neighbour id (22 bits) do not fit one
    32-bit word, so the bucketing passes move (key, neighbour) pairs; the tenants' sketches and answers
    still equal solo runs."""
    rng = np.random.default_rng(12)
    with make_engine(max_vertices=1 << 22) as e:
        specs = TENANTS[:3]
        ids, streams = [], []
        for V, seed, f, gen in specs:
            t = e.add_tenant(V, seed, f)
            ids.append(t)
            streams.append((t, gen()))
        tens, offs, pairs = interleaved_slices(streams, 2, rng)
        e.ingest(tens, offs, pairs)
        res = e.connected_components(ids)
        for (V, seed, f, _), (t, a) in zip(specs, streams):
            sk, labels, ncc, rounds = solo(V, seed, f, a)
            assert e.download(t).tobytes() == sk, t
            assert np.array_equal(res[t].labels, labels), t


def test_query_subsets_and_repeated_queries():
    rng = np.random.default_rng(8)
    with make_engine() as e:
        ids, streams = [], []
        for V, seed, f, gen in TENANTS:
            t = e.add_tenant(V, seed, f)
            ids.append(t)
            streams.append((t, gen()))
        tens, offs, pairs = interleaved_slices(streams, 2, rng)
        e.ingest(tens, offs, pairs)
        full = e.connected_components(ids)
        for subset in ([ids[2]], [ids[4], ids[0]], ids[1:4]):
            part = e.connected_components(subset)
            for t in subset:
                assert np.array_equal(part[t].labels, full[t].labels)
                assert (part[t].num_cc, part[t].rounds) == (full[t].num_cc, full[t].rounds)
        again = e.connected_components(ids, with_labels=False)
        assert all(again[t].num_cc == full[t].num_cc for t in ids)


def test_phases_and_incremental_ingest(restatement):
    """Ingest in phases with a query after each; every phase's answer equals the solo prefix."""
    rng = np.random.default_rng(9)
    with make_engine() as e:
        specs = TENANTS[:3]
        ids = [e.add_tenant(V, seed, f) for V, seed, f, _ in specs]
        streams = [gen() for *_, gen in specs]
        for phase in range(3):
            batch = []
            for t, a in zip(ids, streams):
                cuts = np.linspace(0, len(a), 4).astype(int)
                batch.append((t, a[cuts[phase]:cuts[phase + 1]]))
            rng.shuffle(batch)
            e.ingest_batches(batch)
            res = e.connected_components(ids)
            for (V, seed, f, _), t, a in zip(specs, ids, streams):
                cuts = np.linspace(0, len(a), 4).astype(int)
                prefix = a[: cuts[phase + 1]]
                _, exact = restatement.exact_cc(V, prefix)
                assert np.array_equal(res[t].labels, exact), (phase, t)


def test_admission_by_sketch_bytes_and_slot_reuse():
    per = tenant_bytes(4096)
    budget = 3 * per + per // 2
    with SketchEngine(budget, 8, 1 << 15, 4096, max_batch_edges=1 << 20) as e:
        ids = [e.add_tenant(4096, 100 + i) for i in range(3)]
        used, cap, live = e.memory()
        assert (used, live) == (3 * per, 3) and cap >= budget - 16
        assert e.try_add_tenant(4096, 200) is None           # not admitted: 3.5 tenants of room
        with pytest.raises(gs.GpuSketchError) as err:
            e.add_tenant(4096, 200)
        assert err.value.status == _native.GS_ERR_OOM
        small = e.try_add_tenant(1024, 201)                   # a smaller tenant still fits
        assert small is not None
        # fill the removed tenant's space again: the new tenant starts from zero sketches
        a = gs.er_stream(4096, 0.002, 21, 0.0, 0.0)
        e.ingest_batches([(ids[1], a)])
        e.remove_tenant(ids[1])
        assert e.memory()[2] == 3
        t = e.add_tenant(4096, 300)
        assert not e.download(t).view(np.uint64).any()
        b = gs.er_stream(4096, 0.002, 22, 0.1, 0.5)
        e.ingest_batches([(t, b)])
        sk, labels, ncc, _ = solo(4096, 300, 1.0, b)
        assert e.download(t).tobytes() == sk
        assert e.connected_components([t])[t].num_cc == ncc


def test_tenant_slots_and_vertex_space_limits():
    with SketchEngine(64 << 20, 2, 3000, 2048, max_batch_edges=1 << 20) as e:
        a = e.add_tenant(2048, 1)
        assert e.try_add_tenant(1024, 2) is None               # vertex space: 2048 + 1024 > 3000
        b = e.add_tenant(900, 3)
        assert e.try_add_tenant(16, 4) is None                 # both tenant slots in use
        with pytest.raises(gs.GpuSketchError) as err:
            e.add_tenant(4096, 5)                              # larger than max_tenant_vertices
        assert err.value.status == _native.GS_ERR_BAD_ARG
        e.remove_tenant(a)
        assert e.try_add_tenant(2000, 6) is not None
        del b


def test_bad_records_are_reported_and_skipped():
    with make_engine() as e:
        t0 = e.add_tenant(500, 1)
        t1 = e.add_tenant(800, 2)
        good = gs.er_stream(500, 0.02, 31, 0.0, 0.0)
        bad = np.array([[10, 799]], np.uint32)                 # valid for t1, not for t0
        e.ingest_batches([(t0, good), (t0, bad), (t1, bad)])
        with pytest.raises(gs.GpuSketchError) as err:
            e.synchronize()
        assert err.value.status == _native.GS_ERR_BAD_ARG
        e.synchronize()                                        # the error was reported once
        sk, labels, ncc, _ = solo(500, 1, 1.0, good)
        assert e.download(t0).tobytes() == sk
        sk1, *_ = solo(800, 2, 1.0, bad)
        assert e.download(t1).tobytes() == sk1
        with pytest.raises(gs.GpuSketchError):
            e.ingest([7], [0, 1], bad)                          # tenant 7 is not live


def test_write_binary_per_tenant_reloads(tmp_path):
    with make_engine() as e:
        t = e.add_tenant(1024, 0xC0FFEE)
        a = gs.er_stream(1024, 0.05, 0x5EED0001, 0.10, 0.5)
        e.ingest_batches([(t, a)])
        path = os.path.join(tmp_path, "tenant.bin")
        e.write_binary(t, path)
        with gs.GraphSketch(1024, 0xC0FFEE) as g:
            g.ingest_pairs(a)
            ref = os.path.join(tmp_path, "solo.bin")
            g.write_binary(ref)
        assert open(path, "rb").read() == open(ref, "rb").read()
        with gs.GraphSketch.read_binary(path) as back:
            assert back.connected_components()[1] == e.connected_components([t])[t].num_cc


def test_phase_cuda_graph_matches_eager_and_exact(restatement):
    """Batched phases (device records, one query per phase) with and without CUDA-graph capture."""
    import torch
    from gpusketch_b200.workloads import batched_streams, phase_slices
    streams = batched_streams(12)
    phases = 3
    slices = phase_slices(streams, phases)
    results = []
    for graph in (True, False):
        with SketchEngine(1 << 30, 16, sum(s.V for s in streams), 1 << 14, max_batch_edges=1 << 20) as e:
            ids = [e.add_tenant(s.V, s.sketch_seed) for s in streams]
            per_phase = []
            for p in range(phases):
                parts = [s.records[lo:hi] for s, (lo, hi) in zip(streams, slices[p])]
                offs = np.cumsum([0] + [len(x) for x in parts]).astype(np.uint64)
                d = torch.from_numpy(np.concatenate(parts).astype(np.int32)).cuda()
                per_phase.append(e.phase(ids, offs, d, ids, cuda_graph=graph))
            if graph:
                built, launched = e.graph_stats()
                assert launched == phases and 1 <= built <= phases
            results.append((per_phase, [e.download(t).tobytes() for t in ids]))
    assert results[0] == results[1]
    per_phase, sk = results[0]
    for k, s in enumerate(streams):
        hi = slices[phases - 1][k][1]
        _, exact = restatement.exact_cc(s.V, s.records[:hi])
        assert per_phase[-1][k][0] == len(np.unique(exact)), k
        _, exact1 = restatement.exact_cc(s.V, s.records[:slices[0][k][1]])
        assert per_phase[0][k][0] == len(np.unique(exact1)), k
        sk_solo, *_ = solo(s.V, s.sketch_seed, 1.0, s.records)
        assert sk[k] == sk_solo, k


def test_ingest_slices_pinned_and_pageable():
    import torch
    with make_engine() as e:
        specs = TENANTS[:3]
        ids = [e.add_tenant(V, seed, f) for V, seed, f, _ in specs]
        streams = [gen() for *_, gen in specs]
        batches = []
        for k, (t, a) in enumerate(zip(ids, streams)):
            half = len(a) // 2
            pinned = torch.from_numpy(a[:half].astype(np.int32)).pin_memory()
            batches += [(t, pinned), (t, a[half:])]
        e.ingest_slices(batches[::-1])
        e.ingest_slices([])
        for (V, seed, f, _), t, a in zip(specs, ids, streams):
            sk, *_ = solo(V, seed, f, a)
            assert e.download(t).tobytes() == sk


def test_served_answers_match_solo_runs():
    """Continuous batching with admission: each answer equals the tenant's solo prefix, exactly."""
    from gpusketch_b200.serve import SketchServer
    from gpusketch_b200.workloads import served_trace
    tr = served_trace(num_tenants=8, duration_s=0.25, mean_gap_ms=2.0, query_frac=0.3, log2_batch=(6.0, 11.0),
                      seed=77)
    for i, (V, lg, seed) in enumerate(tr.tenants):       # keep the solo checks small
        v = 1 << (10 + i % 3)
        tr.tenants[i] = (v, 10 + i % 3, seed)
    budget = sum(sorted(tenant_bytes(v) for v, _, _ in tr.tenants)[-3:]) + 4096
    srv = SketchServer(tr, budget, keep_labels=True, keep_sketches=True)
    try:
        stats = srv.run(srv.prepare())
    finally:
        srv.close()
    assert stats.max_live_tenants < len(tr.tenants)     # admission by sketch bytes kept some waiting
    assert stats.answers and stats.updates > 0
    for a in stats.answers:
        V, _, seed = tr.tenants[a.tenant]
        with gs.GraphSketch(V, seed) as g:
            if a.records_before:
                g.ingest_pairs(tr.tenant_records(a.tenant, 0, a.records_before))
            labels, ncc, _ = g.connected_components()
        assert a.num_cc == ncc and np.array_equal(a.labels, labels), a.request
    total = {}
    for r in tr.requests:
        if r.kind == "update":
            total[r.tenant] = total.get(r.tenant, 0) + r.n
    for t, sk in stats.final_sketches.items():
        V, _, seed = tr.tenants[t]
        with gs.GraphSketch(V, seed) as g:
            if total.get(t):
                g.ingest_pairs(tr.tenant_records(t, 0, total[t]))
            assert g.download().tobytes() == sk, t
