"""Seeded synthetic workloads for the multi-tenant engine (batched streams and a served request trace).

Both stand in for independent graph streams of uneven sizes; every stream is reproducible from its
seed, so a tenant's records can be regenerated to check it alone.

batched_streams:  stream i has seed 0x5EED1000+i, V_i = round(2^U(8,14)), average degree
                  d_i ~ U(4,64), Erdos-Renyi G(V_i, d_i/(V_i-1)) in shuffled order with 10% of its
                  edges deleted and half of those re-inserted.
served_trace:     64 tenants with V = round(2^U(10,16)) and R-MAT(0.57,0.19,0.19) edges; requests
                  arrive as a Poisson process (mean gap 2 ms); 10% are connectivity queries, the rest
                  update batches of round(2^U(10,20)) records of one tenant.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .graph import er_stream, rmat_stream

BATCHED_SEED0 = 0x5EED1000
SERVED_SEED = 0x5EED2000


@dataclass
class Stream:
    index: int
    V: int
    sketch_seed: int
    records: np.ndarray  # (n, 2) uint32


def batched_stream_params(count: int = 256, seed0: int = BATCHED_SEED0) -> list[tuple[int, float, int]]:
    """(V, average degree, stream seed) of each batched stream."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed0 + i)
        V = int(round(2.0 ** rng.uniform(8.0, 14.0)))
        d = float(rng.uniform(4.0, 64.0))
        out.append((V, d, seed0 + i))
    return out


def batched_streams(count: int = 256, seed0: int = BATCHED_SEED0, churn: float = 0.10) -> list[Stream]:
    streams = []
    for i, (V, d, seed) in enumerate(batched_stream_params(count, seed0)):
        p = min(1.0, d / (V - 1))
        recs = er_stream(V, p, seed, churn, 0.5)
        streams.append(Stream(i, V, 0xC0FFEE + i, recs))
    return streams


def phase_slices(streams: list[Stream], phases: int):
    """Per phase: (slice tenants order, per-stream [lo, hi) record ranges); stream records split evenly."""
    cuts = [np.linspace(0, len(s.records), phases + 1).astype(np.int64) for s in streams]
    return [[(int(c[p]), int(c[p + 1])) for c in cuts] for p in range(phases)]


@dataclass
class Request:
    t: float             # arrival time (s) from the start of the trace
    tenant: int          # index into ServedTrace.tenants
    kind: str            # "update" or "query"
    first: int = 0       # updates: records [first, first+n) of the tenant's stream
    n: int = 0


@dataclass
class ServedTrace:
    tenants: list[tuple[int, int, int]]  # (V, log2 of the R-MAT space, sketch seed)
    requests: list[Request] = field(default_factory=list)
    duration_s: float = 0.0              # length of the arrival process

    def tenant_records(self, tenant: int, first: int, n: int) -> np.ndarray:
        """Records [first, first+n) of a tenant's stream, on the host (counter-based: any range)."""
        V, lg, seed = self.tenants[tenant]
        r = rmat_stream(lg, n, seed ^ 0xA5A5, first=first)
        return (r % np.uint32(V)).astype(np.uint32)


def served_trace(num_tenants: int = 64, duration_s: float = 1.0, mean_gap_ms: float = 2.0,
                 query_frac: float = 0.10, log2_batch=(10.0, 20.0), seed: int = SERVED_SEED) -> ServedTrace:
    rng = np.random.default_rng(seed)
    tenants = []
    for i in range(num_tenants):
        V = int(round(2.0 ** rng.uniform(10.0, 16.0)))
        tenants.append((V, max(1, math.ceil(math.log2(V))), 0xC0FFEE + 0x100 + i))
    tr = ServedTrace(tenants, duration_s=duration_s)
    cursor = [0] * num_tenants
    t = 0.0
    while True:
        t += rng.exponential(mean_gap_ms / 1000.0)
        if t >= duration_s:
            break
        k = int(rng.integers(num_tenants))
        if rng.random() < query_frac:
            tr.requests.append(Request(t, k, "query"))
        else:
            n = int(round(2.0 ** rng.uniform(*log2_batch)))
            tr.requests.append(Request(t, k, "update", cursor[k], n))
            cursor[k] += n
    return tr


def planted_cut_stream(n_block: int = 8192, p: float = 0.3, cut: int = 3, churn: float = 0.05,
                       seed: int = 0x5EED0003) -> tuple[np.ndarray, np.ndarray]:
    """Two Erdos-Renyi blocks G(n_block, p) on [0, n) and [n, 2n) joined by `cut` random cross edges,
    inserted in random order, then a `churn` share of the edges deleted and re-inserted.
    Returns (records, the planted cut edges)."""
    rng = np.random.default_rng(seed)
    a = er_stream(n_block, p, seed)
    b = er_stream(n_block, p, seed + 1) + np.uint32(n_block)
    cross = np.stack([rng.integers(0, n_block, cut), rng.integers(n_block, 2 * n_block, cut)], 1).astype(np.uint32)
    edges = np.concatenate([a, b, cross])
    edges = edges[rng.permutation(len(edges))]
    k = int(churn * len(edges))
    pick = edges[rng.choice(len(edges), size=k, replace=False)]
    return np.concatenate([edges, pick, pick]), cross
