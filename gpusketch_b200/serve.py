"""Serving loop over the multi-tenant engine: continuous batching of update batches and queries.

Every tenant's sketches stay resident in the engine's device arena.  Requests (update batches of
host records, connectivity queries) are admitted as they arrive:

* a tenant is admitted when its sketch bytes fit in the arena; until then its requests wait;
* each loop iteration coalesces every waiting update batch of admitted tenants (up to a record
  budget) into ONE engine ingest call: one host->device copy, one bucketing pass and one sketch
  update over all of them, the copies of the next slice overlapping the kernels of the previous;
* queries waiting at that point are answered between batches, all of them with ONE multi-tenant
  Boruvka launch;
* a tenant whose last request was served is checkpointed (optional) and removed, freeing its
  arena range for tenants still waiting for admission.

Query latency is measured from arrival (enqueue) to answer.  Because sketches are linear (XOR) and
tenants never share a bucket, each tenant's sketches and answers are independent of how its
requests were batched with other tenants' requests; tests check this against solo runs.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .engine import SketchEngine, tenant_bytes
from .workloads import ServedTrace


@dataclass
class QueryAnswer:
    request: int          # index of the query in the trace
    tenant: int           # trace tenant index
    num_cc: int
    labels: np.ndarray | None
    latency_ms: float
    records_before: int   # the tenant's records ingested before the answer


@dataclass
class ServeStats:
    updates: int = 0
    wall_s: float = 0.0
    ingest_calls: int = 0
    query_launches: int = 0
    max_live_tenants: int = 0
    admissions_deferred: int = 0
    answers: list[QueryAnswer] = field(default_factory=list)
    final_sketches: dict[int, bytes] = field(default_factory=dict)

    def latency_percentiles(self) -> tuple[float, float]:
        lat = np.array([a.latency_ms for a in self.answers]) if self.answers else np.zeros(1)
        return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))

    def latency_summary(self) -> dict:
        lat = np.array([a.latency_ms for a in self.answers]) if self.answers else np.zeros(1)
        return {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                "p99": float(np.percentile(lat, 99)), "max": float(lat.max()), "count": int(len(self.answers)),
                "over_10ms": int((lat > 10.0).sum())}

    @property
    def updates_per_s(self) -> float:
        return self.updates / self.wall_s if self.wall_s > 0 else 0.0


class SketchServer:
    """Replays a ServedTrace against one engine in (scaled) real time."""

    def __init__(self, trace: ServedTrace, sketch_budget_bytes: int, max_batch_records: int = 1 << 23,
                 keep_labels: bool = False, keep_sketches: bool = False, device: int = -1):
        self.trace = trace
        self.max_batch_records = max_batch_records
        self.keep_labels = keep_labels
        self.keep_sketches = keep_sketches
        total_v = sum(v for v, _, _ in trace.tenants)
        max_v = max(v for v, _, _ in trace.tenants)
        self.engine = SketchEngine(sketch_budget_bytes, len(trace.tenants), total_v, max_v, device,
                                   max_batch_edges=max_batch_records)
        self.bytes_needed = [tenant_bytes(v) for v, _, _ in trace.tenants]
        if max(self.bytes_needed) > sketch_budget_bytes:
            raise ValueError("a tenant's sketches are larger than the whole budget")

    def close(self) -> None:
        self.engine.close()

    def prepare(self) -> list[np.ndarray | None]:
        """Host records of every update request (the clients' buffers), generated before the clock starts."""
        return [self.trace.tenant_records(r.tenant, r.first, r.n) if r.kind == "update" else None
                for r in self.trace.requests]

    def run(self, payloads: list[np.ndarray | None], time_scale: float = 1.0) -> ServeStats:
        """Serves every request of the trace; arrivals are paced by the trace times x time_scale.
        A query answers exactly the updates of its tenant that arrived before it."""
        trace, eng = self.trace, self.engine
        reqs = trace.requests
        remaining: dict[int, int] = {}
        for r in reqs:
            remaining[r.tenant] = remaining.get(r.tenant, 0) + 1
        slot: dict[int, int] = {}              # trace tenant -> engine tenant id
        waiting_admission: deque[int] = deque()
        blocked: dict[int, list[int]] = {}     # requests of tenants not admitted yet
        pending: list[int] = []                # requests of admitted tenants, in arrival order
        ingested = {t: 0 for t in remaining}
        stats = ServeStats()
        nxt = 0
        t0 = time.perf_counter()

        def now() -> float:
            return (time.perf_counter() - t0) / time_scale

        def try_admit() -> None:
            admitted = False
            while waiting_admission:
                t = waiting_admission[0]
                V, _, seed = trace.tenants[t]
                e = eng.try_add_tenant(V, seed)
                if e is None:
                    stats.admissions_deferred += 1
                    break
                waiting_admission.popleft()
                slot[t] = e
                pending.extend(blocked.pop(t))
                admitted = True
                stats.max_live_tenants = max(stats.max_live_tenants, eng.memory()[2])
            if admitted:
                pending.sort()

        def retire(t: int) -> None:
            if self.keep_sketches:
                stats.final_sketches[t] = eng.download(slot[t]).tobytes()
            eng.remove_tenant(slot.pop(t))

        while nxt < len(reqs) or pending or blocked:
            # ---- arrivals ----
            cur = now()
            while nxt < len(reqs) and reqs[nxt].t <= cur:
                r = reqs[nxt]
                if r.tenant in slot:
                    pending.append(nxt)
                else:
                    if r.tenant not in blocked:
                        blocked[r.tenant] = []
                        waiting_admission.append(r.tenant)
                    blocked[r.tenant].append(nxt)
                nxt += 1
            try_admit()
            if not pending:
                if nxt < len(reqs):
                    wait = reqs[nxt].t - now()
                    if wait > 0:
                        time.sleep(min(wait * time_scale, 0.001))
                continue
            # ---- pick this iteration's work in arrival order: every update batch that fits the record
            #      budget and every query; a tenant's later requests wait behind its query or behind
            #      its own deferred update, so each query sees exactly its tenant's earlier updates ----
            batch, queries, keep, hold, total = [], [], [], set(), 0
            for i in pending:
                r = reqs[i]
                if r.tenant in hold:
                    keep.append(i)
                elif r.kind == "query":
                    queries.append(i)
                    hold.add(r.tenant)
                elif not batch or total + r.n <= self.max_batch_records:
                    batch.append(i)
                    total += r.n
                else:
                    keep.append(i)
                    hold.add(r.tenant)
            pending = keep
            done_tenants = []
            # ---- one coalesced ingest of the chosen update batches ----
            if batch:
                eng.ingest_slices([(slot[reqs[i].tenant], payloads[i]) for i in batch])
                stats.ingest_calls += 1
                stats.updates += total
                for i in batch:
                    t = reqs[i].tenant
                    ingested[t] += reqs[i].n
                    remaining[t] -= 1
                    if remaining[t] == 0:
                        done_tenants.append(t)
            # ---- queries between batches: one multi-tenant Boruvka launch ----
            if queries:
                tens = sorted({reqs[i].tenant for i in queries})
                res = eng.connected_components([slot[t] for t in tens], with_labels=self.keep_labels)
                stats.query_launches += 1
                answered = now()
                for i in queries:
                    t = reqs[i].tenant
                    r = res[slot[t]]
                    stats.answers.append(QueryAnswer(i, t, r.num_cc, r.labels.copy() if r.labels is not None else None,
                                                     1000.0 * (answered - reqs[i].t), ingested[t]))
                    remaining[t] -= 1
                    if remaining[t] == 0:
                        done_tenants.append(t)
            for t in done_tenants:
                retire(t)
            if done_tenants:
                try_admit()
        eng.synchronize()
        stats.wall_s = time.perf_counter() - t0
        return stats


class PlainServer:
    """The same trace on the single-graph path: one GraphSketch per tenant, requests served one at a
    time in arrival order (an ingest call per update batch, a Boruvka launch per query)."""

    def __init__(self, trace: ServedTrace, device: int = -1, max_batch_edges: int = 1 << 20):
        from .graph import GraphSketch
        self.trace = trace
        self.handles = {}
        for t in sorted({r.tenant for r in trace.requests}):
            V, _, seed = trace.tenants[t]
            self.handles[t] = GraphSketch(V, seed, device=device, max_batch_edges=max_batch_edges)

    def close(self) -> None:
        for h in self.handles.values():
            h.close()

    def run(self, payloads: list[np.ndarray | None], time_scale: float = 1.0, keep_labels: bool = False) -> ServeStats:
        reqs = self.trace.requests
        ingested = {t: 0 for t in self.handles}
        stats = ServeStats()
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            wait = r.t * time_scale - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            h = self.handles[r.tenant]
            if r.kind == "update":
                h.ingest_pairs(payloads[i])
                stats.ingest_calls += 1
                stats.updates += r.n
                ingested[r.tenant] += r.n
            else:
                labels, ncc, _ = h.connected_components()
                stats.query_launches += 1
                lat = 1000.0 * ((time.perf_counter() - t0) / time_scale - r.t)
                stats.answers.append(QueryAnswer(i, r.tenant, ncc, labels if keep_labels else None, lat,
                                                 ingested[r.tenant]))
        for h in self.handles.values():
            h.synchronize()
        stats.wall_s = time.perf_counter() - t0
        return stats
