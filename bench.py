#!/usr/bin/env python
"""Benchmark of the large-ingest workload: R-MAT(0.57,0.19,0.19,0.05) over V=2^17 vertices, 2^30 edge
updates (~12% deletions of earlier inserts) generated on the device from a seed, with a connected-
components query after every 2^27 updates (8 ingest phases + 8 queries per step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gs|reference]

One step = clear the V sketches, then 8 x (ingest 2^27 records + connected_components()).  The records
(8 GiB per GPU) are resident in HBM before timing and larger than L2.  `value` is the edge-update rate
of the K timed steps (CUDA events on the stream the library launches on; max over ranks); `e2e` is the
same workload through the C ABI from pinned host buffers (H2D inside the timed region) with the
component labels copied back after every query; each phase's query is queued (gs_connected_components_async)
and the next phase's records are queued behind it (gs_ingest_pairs_async) before its answer is collected.  N > 1 ranks run independent replicas (seed + rank).
`--impl reference` times the reference's own CPU CCSketchAlg (compiled from its sources into
oracle/_ref) on a bounded sample of the same stream with every host thread.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from gpusketch_b200.replicas import (barrier as rank_barrier, env_rank, max_over_ranks as rank_max,
                                     replica_seed, sum_over_ranks, whole_job_rate)

V_LOG2 = 17
STREAM_SEED = 0x5EED0002
SKETCH_SEED = 0xC0FFEE
METRIC = "edge updates/sec"
UNIT = "edge_updates/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gs", "reference"], default="gs")
    ap.add_argument("--updates-log2", type=int, default=30)
    ap.add_argument("--phase-log2", type=int, default=27)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default launch parameters")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target wall time of the CPU sample")
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-stream batched engine comparison")
    ap.add_argument("--no-served", action="store_true", help="skip the 64-tenant served trace")
    ap.add_argument("--no-mincut", action="store_true", help="skip the planted-cut min-cut workload")
    ap.add_argument("--batched-streams", type=int, default=256)
    ap.add_argument("--batched-phases", type=int, default=4)
    ap.add_argument("--served-seconds", type=float, default=10.0, help="length of the x1 served request trace")
    ap.add_argument("--served-loads", default="1,4,16,64", help="offered-load factors of the served sweep")
    ap.add_argument("--no-dropin", action="store_true", help="skip the stream-file and C++ drop-in sub-lines")
    return ap.parse_args()


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


KERNEL_SOURCES = ("gpusketch_b200/csrc/gs_ingest.cu", "gpusketch_b200/csrc/gs_common.cuh")


def kernel_source_sha16() -> str:
    """sha256 (first 16 hex digits) of the sketch-update kernel's sources with comments and blank
    lines removed, as the ncu summaries record it: a committed capture describes the current kernel
    only when the two agree (an edit of a comment leaves the code, and the capture, current)."""
    import hashlib
    import re
    h = hashlib.sha256()
    for rel in KERNEL_SOURCES:
        with open(os.path.join(ROOT, rel), encoding="utf-8") as f:
            text = f.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        lines = (re.sub(r"//.*$", "", ln).rstrip() for ln in text.splitlines())
        h.update("\n".join(ln for ln in lines if ln).encode())
    return h.hexdigest()[:16]


def _profile_field(name: str, key: str):
    """(value, source sha16 recorded with it) from a committed ncu summary in profiles/."""
    value = sha = None
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith(key + ":"):
                value = float(line.split(":", 1)[1])
            elif line.startswith("source_sha256_16:"):
                sha = line.split(":", 1)[1].strip()
    except OSError:
        pass
    return value, sha


def ncu_issue_per_launch():
    """warp instructions of one full-size ingest launch from the committed ncu summary, and whether that
    capture ran the current kernel sources."""
    v, sha = _profile_field("k_ingest_rmat17_issue.txt", "warp_instructions_per_full_launch")
    return v, sha == kernel_source_sha16()


def ncu_smem_per_launch():
    """shared-memory wavefronts of one full-size ingest launch from the committed ncu summary, and
    whether that capture ran the current kernel sources."""
    v, sha = _profile_field("k_ingest_rmat17_issue.txt", "smem_wavefronts_per_full_launch")
    return v, sha == kernel_source_sha16()


def ncu_traffic_per_launch():
    """dram bytes read+write of one full-size ingest launch from the committed ncu summary, and whether
    that capture ran the current kernel sources."""
    v, sha = _profile_field("k_ingest_rmat17_traffic.txt", "traffic_bytes_per_full_launch")
    return v, sha == kernel_source_sha16()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].isdigit():
                    rows.append(f)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [int(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def cpu_baseline(pairs_host, V, phase, target_s, threads=None):
    """The reference's CCSketchAlg (oracle/_ref, its own sources) on a bounded prefix of the stream:
    records bucketed by endpoint into reference-sized batches (outside the timing), then
    apply_update_batch from T std::threads, plus one connected_components() pro-rated per `phase`."""
    import numpy as np
    from oracle import RefCC, bucket_by_vertex

    T = threads or len(os.sched_getaffinity(0))
    ref = RefCC(V, SKETCH_SEED, 1.0, workers=T)
    batch = int(ref.L.gsref_cc_desired_batch(ref.h))
    # calibrate on 2^20 records, then size the sample to ~target_s of ingest
    cal = np.ascontiguousarray(pairs_host[: 1 << 20])
    b = bucket_by_vertex(cal, V, batch)
    t0 = time.perf_counter()
    ref.ingest_batches(*b, threads=T)
    rate0 = len(cal) / (time.perf_counter() - t0)
    n = int(min(len(pairs_host), max(1 << 20, rate0 * target_s)))
    n = 1 << (n.bit_length() - 1)
    sample = np.ascontiguousarray(pairs_host[:n])
    b = bucket_by_vertex(sample, V, batch)
    t0 = time.perf_counter()
    ref.ingest_batches(*b, threads=T)
    t_ing = time.perf_counter() - t0
    t0 = time.perf_counter()
    labels, ncc, rounds = ref.connected_components()
    t_cc = time.perf_counter() - t0
    ref.close()
    rate = n / (t_ing + t_cc * n / phase)
    return {"value": rate, "unit": UNIT, "cores": T, "kind": "reference",
            "sample": f"first 2^{n.bit_length() - 1} records of the same R-MAT stream, bucketed by endpoint into "
                      f"{batch}-dst batches (untimed), CCSketchAlg::apply_update_batch from {T} threads "
                      f"({t_ing:.2f} s) + one connected_components() ({t_cc:.2f} s) pro-rated at one per 2^"
                      f"{phase.bit_length() - 1} records"}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    import numpy as np
    import gpusketch_b200 as gs
    from oracle import RefCC, bucket_by_vertex, ref_available

    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libgsref.so was not built"}))
        return
    V = 1 << V_LOG2
    phase = 1 << args.phase_log2
    T = len(os.sched_getaffinity(0))
    # size one step to a bounded sample: calibrate, then ~target s per step
    n_total = 1 << min(args.updates_log2, 26)
    pairs = gs.rmat_stream(V_LOG2, n_total, STREAM_SEED)
    ref = RefCC(V, SKETCH_SEED, 1.0, workers=T)
    batch = int(ref.L.gsref_cc_desired_batch(ref.h))
    cal = bucket_by_vertex(pairs[: 1 << 20], V, batch)
    t0 = time.perf_counter()
    ref.ingest_batches(*cal, threads=T)
    rate0 = (1 << 20) / (time.perf_counter() - t0)
    budget = 150.0 / max(1, args.steps + args.warmup)  # the whole run within a few minutes
    n = int(min(n_total, max(1 << 20, rate0 * budget)))
    n = 1 << (n.bit_length() - 1)
    b = bucket_by_vertex(pairs[:n], V, batch)
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        ref.ingest_batches(*b, threads=T)
        t1 = time.perf_counter()
        ref.connected_components()
        t2 = time.perf_counter()
        if it >= args.warmup:
            times.append((t1 - t0) + (t2 - t1) * n / phase)
    ref.close()
    sec = sum(times) / len(times)
    value = n / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "large_ingest_rmat17", "V": V, "updates_per_step": n,
                   "phase_updates": phase, "sample": True},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": T, "kind": "reference",
                         "sample": f"2^{n.bit_length() - 1} records per step of the R-MAT stream, bucketed by "
                                   f"endpoint (untimed); CCSketchAlg::apply_update_batch from {T} threads + "
                                   f"connected_components() pro-rated at one per 2^{args.phase_log2} records"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_batched(args, dev, steps, warmup):
    """256 independent ER streams (seeds 0x5EED1000+i, V = round(2^U(8,14)), degree U(4,64), 10% churn)
    in `phases` phases.  Engine: one gs_engine_phase per phase (device-resident slices of every stream,
    then one Boruvka launch over all 256 tenants), recorded and launched as one CUDA graph.  Plain: the
    single-graph path, one GraphSketch per stream, an ingest call and a connected_components() call per
    stream per phase.  Both from device-resident records; wall time with the device idle on both sides
    (each call returns after its work finished)."""
    import numpy as np
    import torch
    import gpusketch_b200 as gs
    from gpusketch_b200.autotune import autotune_engine
    from gpusketch_b200.engine import SketchEngine, tenant_bytes
    from gpusketch_b200.workloads import batched_streams, phase_slices

    streams = batched_streams(args.batched_streams)
    P = args.batched_phases
    slices = phase_slices(streams, P)
    total = sum(len(s.records) for s in streams)
    d_phase, offs = [], []
    for p in range(P):
        parts = [s.records[lo:hi] for s, (lo, hi) in zip(streams, slices[p])]
        offs.append(np.cumsum([0] + [len(x) for x in parts]).astype(np.uint64))
        d_phase.append(torch.from_numpy(np.concatenate(parts).astype(np.int32)).to(dev))
    budget = sum(tenant_bytes(s.V) for s in streams) + (64 << 20)
    eng = SketchEngine(budget, len(streams), sum(s.V for s in streams), 1 << 14, device=dev.index)
    ids = [eng.add_tenant(s.V, s.sketch_seed) for s in streams]
    tune = autotune_engine(eng, ids, offs[0], d_phase[0])
    for t in ids:
        eng.clear_tenant(t)

    def engine_step(graph=True):
        for t in ids:
            eng.clear_tenant(t)
        out = []
        for p in range(P):
            out.append(eng.phase(ids, offs[p], d_phase[p], ids, cuda_graph=graph))
        return out

    def timed(fn, n):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = None
        for _ in range(n):
            res = fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / n, res

    for _ in range(warmup):
        engine_step()
    eng_s, eng_res = timed(engine_step, steps)
    eng.profile_enable(True)  # per-kernel-class split from the eager phases (graphs carry no timing events)
    eager_s, eager_res = timed(lambda: engine_step(False), steps)
    prof = eng.profile_read()
    eng.profile_enable(False)
    built, launched = eng.graph_stats()
    used = eng.memory()[0]
    eng.close()

    handles = [gs.GraphSketch(s.V, s.sketch_seed, device=dev.index, max_batch_edges=1 << 20) for s in streams]

    def plain_step():
        for h in handles:
            h.clear()
        out = []
        for p in range(P):
            res = {}
            d, o = d_phase[p], offs[p]
            for k, h in enumerate(handles):
                h.ingest_pairs(d[int(o[k]):int(o[k + 1])])
                res[ids[k]] = h.connected_components()[1]
            out.append(res)
        return out

    plain_step()
    plain_runs = []
    for _ in range(3):
        t, plain_res = timed(plain_step, 1)
        plain_runs.append(t)
    plain_s = statistics.median(plain_runs)
    for h in handles:
        h.close()
    agree = all(plain_res[p][t] == eng_res[p][t][0] == eager_res[p][t][0] for p in range(P) for t in ids)
    return {
        "workload": f"batched_{len(streams)}_er_streams", "scope": "one GPU (rank 0)", "streams": len(streams), "phases": P,
        "updates_per_step": total, "vertices": sum(s.V for s in streams), "sketch_bytes": used,
        "engine_value": total / eng_s, "engine_eager_value": total / eager_s, "plain_value": total / plain_s,
        "unit": UNIT, "speedup_vs_plain": plain_s / eng_s, "engine_ms_per_step": 1e3 * eng_s,
        "engine_eager_ms_per_step": 1e3 * eager_s, "plain_ms_per_step": 1e3 * plain_s,
        "plain_ms_per_step_runs": [1e3 * t for t in plain_runs],
        "engine_eager_split_ms_per_step": {k: prof[k] / steps for k in ("ingest_ms", "bucket_ms", "query_ms")},
        "cuda_graphs": {"instantiated": built, "launched": launched},
        "tuning": tune, "answers_agree": agree,
        "timing": "wall clock per step around synchronous calls, device idle on both sides; plain: median of 3 steps",
    }


def _served_once(tr, dev, with_plain: bool) -> dict:
    import torch
    from gpusketch_b200.engine import tenant_bytes
    from gpusketch_b200.serve import PlainServer, SketchServer
    need = sum(tenant_bytes(v) for v, _, _ in tr.tenants)
    srv = SketchServer(tr, need + (256 << 20), device=dev.index)
    host = srv.prepare()
    payloads = [torch.from_numpy(a.astype("int32")).pin_memory() if a is not None else None for a in host]
    del host
    srv.run(payloads, time_scale=0.05)  # warm-up pass 20x faster than real time; every tenant retires
    st = srv.run(payloads)
    srv.close()
    offered = sum(r.n for r in tr.requests if r.kind == "update")
    out = {"requests": len(tr.requests), "queries": len(st.answers), "offered_updates": offered,
           "offered_updates_per_s": offered / tr.duration_s, "updates_per_s": st.updates_per_s,
           "query_latency_ms": st.latency_summary(), "ingest_calls": st.ingest_calls,
           "query_launches": st.query_launches, "wall_s": st.wall_s, "max_live_tenants": st.max_live_tenants,
           "sketch_bytes_needed": need}
    if with_plain:
        plain = PlainServer(tr, device=dev.index)
        pst = plain.run(payloads)
        plain.close()
        out["plain_query_latency_ms"] = pst.latency_summary()
        out["plain_updates_per_s"] = pst.updates_per_s
        out["plain_wall_s"] = pst.wall_s
    del payloads
    return out


def run_served(args, dev):
    """64 tenants (V = round(2^U(10,16)), R-MAT records), Poisson arrivals, update batches of
    round(2^U(10,20)) records from page-locked host buffers, 10% connectivity queries; replayed in real
    time by the continuous-batching server.  The offered load is swept: at load x f the mean gap is
    2/f ms and the trace lasts served_seconds/f, so every point offers the same records and about as
    many queries (about 500 at 10 s).  The plain per-tenant server replays the x1 trace."""
    from gpusketch_b200.workloads import served_trace

    loads = [float(x) for x in args.served_loads.split(",")]
    sweep = []
    for f in loads:
        tr = served_trace(64, args.served_seconds / f, mean_gap_ms=2.0 / f)
        point = _served_once(tr, dev, with_plain=(f == 1.0))
        point["load"] = f
        point["trace_seconds"] = tr.duration_s
        sweep.append(point)
    base = next((p for p in sweep if p["load"] == 1.0), sweep[0])
    crossing = next((p["load"] for p in sweep if p["query_latency_ms"]["p99"] > 10.0), None)
    return {
        "workload": "served_64_tenants_rmat", "scope": "one GPU (rank 0)", "tenants": 64,
        "trace_seconds": args.served_seconds, "requests": base["requests"], "queries": base["queries"],
        "offered_updates": base["offered_updates"], "query_latency_ms": base["query_latency_ms"],
        "updates_per_s": base["updates_per_s"], "plain_query_latency_ms": base.get("plain_query_latency_ms"),
        "plain_updates_per_s": base.get("plain_updates_per_s"), "ingest_calls": base["ingest_calls"],
        "query_launches": base["query_launches"], "wall_s": base["wall_s"],
        "max_live_tenants": base["max_live_tenants"], "sketch_bytes_needed": base["sketch_bytes_needed"],
        "load_sweep": [{k: p[k] for k in ("load", "trace_seconds", "offered_updates_per_s", "updates_per_s",
                                          "queries", "query_latency_ms", "wall_s")} for p in sweep],
        "p99_over_10ms_from_load": crossing,
        "latency": "enqueue (trace arrival time) to answer, wall clock",
    }


def run_dropin(args, dev):
    """Stream files and the reference-facing C++ classes, one GPU:
    * file_ingest: a 2^27-record binary stream file (the reference's format, 1.2 GB, R-MAT V=2^17) read by
      the library (gs_ingest_stream_file: parallel pread into the page-locked ring, device decode),
      timed from the call to the end of the device work; the file is in the page cache;
    * reference_tool: the reference's own tools/cuda_process_stream.cu, compiled unchanged against the
      drop-in headers, on the same file: its "Updates per second" line (GraphSketchDriver ->
      CCGPUSketchAlg, insertion time including the final flush);
    * apply_update_batch: the reference's worker path on the first 2^26 records - per-vertex batches of
      get_desired_updates_per_batch() destinations (grouped on the host, untimed) handed to
      CCGPUSketchAlg::apply_update_batch from 8 worker threads, then flush_buffers and
      connected_components() (timed)."""
    import tempfile
    import numpy as np
    import torch
    import gpusketch_b200 as gs
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from stream_file import write_stream_file

    out = {"scope": "one GPU (rank 0)"}
    V = 1 << V_LOG2
    n = 1 << 27
    d = torch.empty((n, 2), dtype=torch.int32, device=dev)
    gs.rmat_stream(V_LOG2, n, STREAM_SEED, out=d)
    host = d.cpu().numpy().view(np.uint32)
    del d
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "rmat17_2p27.data")
        write_stream_file(path, V, host, types=np.zeros(n, np.uint8))
        small = os.path.join(tmp, "rmat17_2p26.data")
        write_stream_file(small, V, host[: 1 << 26], types=np.zeros(1 << 26, np.uint8))
        del host
        fbytes = os.path.getsize(path)
        with gs.GraphSketch(V, SKETCH_SEED, device=dev.index) as g:
            g.prepare_host_input(n)                      # the page-locked ring for full-size slices
            g.ingest_stream_file(path)                   # warm-up: full-size scratch, decode buffer, page cache
            g.clear()
            g.synchronize()
            rates = []
            for _ in range(3):
                g.clear()
                g.synchronize()
                t0 = time.perf_counter()
                got = g.ingest_stream_file(path)
                g.synchronize()
                rates.append(got / (time.perf_counter() - t0))
        r = statistics.median(rates)
        out["file_ingest"] = {"records": n, "file_bytes": fbytes, "updates_per_s": r, "file_gb_per_s": r * 9 / 1e9,
                              "runs": rates, "timing": "wall clock, call to end of device work, median of 3"}
        tool = os.path.join(ROOT, "oracle", "_ref", "cuda_process_stream")
        if os.path.exists(tool):
            res = subprocess.run([tool, path, "8", "2"], capture_output=True, text=True, timeout=600, cwd=tmp)
            line = [l for l in res.stdout.splitlines() if l.startswith("Updates per second:")]
            cc = [l for l in res.stdout.splitlines() if l.startswith("Connected Components:")]
            out["reference_tool"] = {"tool": "tools/cuda_process_stream.cu (unchanged) + drop-in headers",
                                     "rc": res.returncode,
                                     "updates_per_s": float(line[0].split(":")[1]) if line else None,
                                     "connected_components": int(cc[0].split(":")[1]) if cc else None}
        demo = os.path.join(ROOT, "gpusketch_b200", "_build", "cc_dropin_demo")
        if os.path.exists(demo):
            res = subprocess.run([demo, small, str(SKETCH_SEED), "-", "1", "batches"], capture_output=True, text=True,
                                 timeout=900, cwd=tmp)
            line = [l for l in res.stdout.splitlines() if l.startswith("updates=")]
            f = dict(kv.split("=") for kv in line[0].split()) if line else {}
            out["apply_update_batch"] = {"records": 1 << 26, "rc": res.returncode,
                                         "updates_per_s": float(f["updates_per_sec"]) if f else None,
                                         "batches": int(f["batches"]) if f else None,
                                         "seconds": float(f["seconds"]) if f else None,
                                         "path": "CCGPUSketchAlg::apply_update_batch x 8 threads + flush + CC"}
    return out


def run_mincut(args, dev):
    """k-connectivity / min cut: V=2^14 as two ER blocks of 8192 (p=0.3) joined by 3 planted edges,
    inserted in random order then 5% deleted and re-inserted (~22M records); k=4 forests per level over
    4 sketched subgraph levels (tags get_index_depth(e, seed, L-1), L = 1 + 2 log2 V).  Timed: the
    tagged ingest of the device-resident records, then the level-by-level min-cut driver."""
    import numpy as np
    import torch
    import gpusketch_b200 as gs
    from gpusketch_b200.workloads import planted_cut_stream
    n = 8192
    recs, _ = planted_cut_stream(n)
    V = 2 * n
    L = 1 + 2 * int(np.log2(V))
    # the sketch size the reference's min-cut tool uses: sketches_factor = reduced_k
    # (tools/min_cut.cu:95-96,156), 51 samples per sketch at V=2^14
    k_tool = int(np.ceil(np.log2(V) / 0.75 ** 2))
    reduced_k = (k_tool / np.log2(V)) * 1.5
    d = torch.from_numpy(recs.astype(np.int32)).to(dev)
    g = gs.GraphSketch(V, 0x5EED0003, sketches_factor=reduced_k, num_levels=4, num_subgraphs=L, device=dev.index,
                       max_batch_edges=1 << 25)
    g.ingest_pairs(d)            # warm-up of the same work, then cleared
    g.min_cut(4)
    g.clear()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g.ingest_pairs(d)
    g.synchronize()
    t1 = time.perf_counter()
    value, level, cut_at, side = g.min_cut(4)
    t2 = time.perf_counter()
    g.close()
    return {"workload": "mincut_planted_v16384", "scope": "one GPU (rank 0)", "records": int(len(recs)),
            "levels": 4, "k": 4, "num_subgraphs": L, "sketches_factor": reduced_k,
            "sketch_columns": gs.geometry_for(V, reduced_k).num_columns,
            "sketch_bytes_per_vertex_level": gs.geometry_for(V, reduced_k).bytes_per_vertex,
            "ingest_updates_per_s": len(recs) / (t1 - t0),
            "ingest_ms": 1e3 * (t1 - t0), "min_cut_ms": 1e3 * (t2 - t1), "value": value, "expected": 3,
            "level": level, "cut_at_level": cut_at,
            "timing": "wall clock around synchronous calls, device idle on both sides"}


def run_gs(args):
    import numpy as np
    import torch
    import gpusketch_b200 as gs

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    V = 1 << V_LOG2
    U = 1 << args.updates_log2
    phase = 1 << args.phase_log2
    P = U // phase
    stream_seed = replica_seed(STREAM_SEED, rank)
    dev = torch.device("cuda", local)

    d_in = torch.empty((U, 2), dtype=torch.int32, device=dev)
    gs.rmat_stream(V_LOG2, U, stream_seed, out=d_in)
    torch.cuda.synchronize()

    g = gs.GraphSketch(V, replica_seed(SKETCH_SEED, rank), device=local, max_batch_edges=phase)
    ts = torch.cuda.current_stream()
    g.set_stream(ts)
    geo = g.geometry
    # launch parameters picked by the autotuner on the first phase's records (untimed set-up)
    from gpusketch_b200.autotune import autotune
    tune_table = []
    if args.no_autotune:
        from gpusketch_b200.autotune import get_tuning
        tuning = get_tuning(g)
    else:
        tuning = autotune(g, d_in[: min(phase, 1 << 25)], table=tune_table)
    g.clear()

    def step(src):
        # each phase's query is queued behind its records and the next phase's records behind the
        # query before its answer (labels, component count) is collected, so the device never idles
        # while the host collects an answer; every phase is still ingested, queried and answered
        g.clear()
        g.ingest_pairs(src[0:phase])
        for p in range(P):
            g.connected_components_async()
            if p + 1 < P:
                g.ingest_pairs(src[(p + 1) * phase:(p + 2) * phase])
            g.query_wait()

    def barrier():
        rank_barrier(dist)

    def max_over_ranks(x: float) -> float:
        return rank_max(x, dist, dev)

    for _ in range(args.warmup):
        step(d_in)
    torch.cuda.synchronize()
    g.profile_enable(True)
    barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(ts)
        for _ in range(args.steps):
            step(d_in)
        end.record(ts)
        torch.cuda.synchronize()
    barrier()
    ms = start.elapsed_time(end)
    prof = g.profile_read()
    clocks = clk.summary()
    ms_max = max_over_ranks(ms)
    ms_per_step = ms_max / args.steps
    value = whole_job_rate(sum_over_ranks(U * args.steps, dist, dev), ms_max)

    # roofline of the dominant kernel (the sketch update), per launch: B_edge = 8 + 2*V*S_v/U_phase
    # bytes per edge update (the read half dropped for the first phase of a step, whose sketches are 0)
    Sv = geo.bytes_per_vertex
    alg_step = 8.0 * U + V * Sv * (2 * P - 1)
    alg_per_launch = alg_step / P
    launches = max(1, prof["ingest_launches"])
    ingest_ms_avg = prof["ingest_ms"] / launches
    achieved = alg_per_launch / (ingest_ms_avg / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic, traffic_current = ncu_traffic_per_launch()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_source": "committed ncu capture (profiles/k_ingest_rmat17_traffic.txt)",
                "traffic_capture_matches_source": traffic_current, "peak_source": peak_kind,
                "kernel": "k_ingest_packed (sketch update)", "alg_bytes_per_launch": alg_per_launch,
                "avg_launch_ms": ingest_ms_avg, "path_frac": value / world * (alg_step / U) / 1e9 / peak}
    # the sketch update is bound by instruction issue: its measured warp instructions per launch
    # (one-pass ncu count of this workload's launch) against 4 schedulers x SMs x the sampled SM clock
    issue = None
    inst, inst_current = ncu_issue_per_launch()
    if inst is not None and V == (1 << 17) and phase == (1 << 27) and clocks.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        ach = inst / (ingest_ms_avg / 1e3)
        pk = 4.0 * sms * clocks["sm_mhz"] * 1e6
        issue = {"bound": "issue", "achieved": ach, "peak": pk, "unit": "warp_inst/s", "frac": ach / pk,
                 "inst_per_launch": inst, "inst_source": "committed ncu capture (profiles/k_ingest_rmat17_issue.txt)",
                 "inst_capture_matches_source": inst_current, "kernel": "k_ingest_packed (sketch update)",
                 "peak_source": f"4 schedulers x {sms} SMs x median sampled SM clock"}
    # ... and by shared-memory bandwidth: every (record, column) reads and writes a 16-byte row and every
    # record is broadcast from the warp's stage; one wavefront (128 B) per SM and clock is the peak
    smem = None
    wf, wf_current = ncu_smem_per_launch()
    if wf is not None and V == (1 << 17) and phase == (1 << 27) and clocks.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        ach = wf / (ingest_ms_avg / 1e3)
        pk = 1.0 * sms * clocks["sm_mhz"] * 1e6
        smem = {"bound": "shared-memory wavefronts", "achieved": ach, "peak": pk, "unit": "wavefronts/s",
                "frac": ach / pk, "wavefronts_per_launch": wf,
                "wavefront_source": "committed ncu capture (profiles/k_ingest_rmat17_issue.txt)",
                "wavefront_capture_matches_source": wf_current, "kernel": "k_ingest_packed (sketch update)",
                "peak_source": f"one 128-byte wavefront per SM and clock x {sms} SMs x median sampled SM clock"}
    split = {"ingest_ms_per_step": prof["ingest_ms"] / args.steps, "bucket_ms_per_step": prof["bucket_ms"] / args.steps,
             "query_ms_per_step": prof["query_ms"] / args.steps}

    e2e = None
    if not args.no_e2e:
        h_in = torch.empty((U, 2), dtype=torch.int32, pin_memory=True)
        h_in.copy_(d_in)
        labels_host = torch.empty(V, dtype=torch.int32, pin_memory=True)

        def run_e2e(steps):
            # each phase's query is queued behind its records, then the next records (copies included;
            # after a step's last phase the next step's clear and first records) are queued behind the
            # query before its answer is collected, so the copy engine never waits for a query
            g.clear()
            g.ingest_pairs_async(h_in[0:phase])                    # host pinned -> H2D inside the library
            for s in range(steps):
                for p in range(P):
                    g.connected_components_async()
                    if p + 1 < P:
                        g.ingest_pairs_async(h_in[(p + 1) * phase:(p + 2) * phase])
                    elif s + 1 < steps:
                        g.clear()
                        g.ingest_pairs_async(h_in[0:phase])
                    labels, _, _ = g.query_wait()                  # labels copied back to the host
        run_e2e(max(1, args.warmup))
        torch.cuda.synchronize()
        barrier()
        e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_start.record(ts)
        run_e2e(args.steps)
        e_end.record(ts)
        torch.cuda.synchronize()
        barrier()
        ems = max_over_ranks(e_start.elapsed_time(e_end))
        e2e = {"value": whole_job_rate(world * U * args.steps, ems), "unit": UNIT, "h2d_bytes_per_step": U * 8,
               "d2h_bytes_per_step": P * V * 4, "ms_per_step": ems / args.steps}
        del h_in

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sample = d_in[: 1 << 26].cpu().numpy().astype(np.uint32)
            cpu = cpu_baseline(sample, V, phase, args.cpu_seconds)
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "reference", "sample": f"failed: {exc}"}

    g.close()
    del d_in
    torch.cuda.empty_cache()
    # the one-GPU sub-lines (min cut, drop-in, batched, served) run at N=1 only: at N>1 they would
    # hold every GPU for a minute of measurements the scaling line does not use
    batched = served = mincut = dropin = None
    if not args.no_mincut and world == 1:
        mincut = run_mincut(args, dev)
    if not args.no_dropin and world == 1:
        try:
            dropin = run_dropin(args, dev)
        except Exception as exc:  # a sub-line, never required
            dropin = {"error": str(exc)}
    if not args.no_batched and world == 1:
        batched = run_batched(args, dev, max(1, args.steps), max(1, args.warmup))
    if not args.no_served and world == 1:
        served = run_served(args, dev)
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "large_ingest_rmat17", "V": V, "updates_per_step": U, "phase_updates": phase,
                   "cc_queries_per_step": P, "rmat": [0.57, 0.19, 0.19, 0.05], "delete_frac": 0.12,
                   "stream_seed": f"{STREAM_SEED:#x}+rank", "sketch_seed": f"{SKETCH_SEED:#x}+rank",
                   "sketch_bytes_per_vertex": Sv, "l2": "inputs larger than L2 (8 GiB of records per GPU)",
                   "parallelism": f"replicas x{world}", "tuning": tuning},
        "roofline": roofline, "issue_roofline": issue, "smem_roofline": smem, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": prof["kernel_launches"],
        "clocks": clocks, "kernel_split": split, "batched": batched, "served": served,
        "mincut": mincut, "dropin": dropin,
    }
    if os.environ.get("GS_BENCH_TUNE_TABLE"):
        line["tune_table"] = tune_table
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gs(args)


if __name__ == "__main__":
    main()
