"""SketchEngine: many independent connected-components graphs (tenants) resident on one GPU.

Binds the gs_engine_* entry points of include/gpusketch.h.  Every tenant's sketches are bit-identical
to a GraphSketch (and the reference's CCSketchAlg) with the same num_vertices, seed and
sketches_factor fed the same records; an ingest call carries record slices of many tenants and
runs the bucketing and the sketch update once for all of them, and a query answers
connected_components() for a list of tenants with one device Boruvka launch.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._native import GS_ERR_OOM, GS_PHASE_CUDA_GRAPH, GpuSketchError, GsEngineConfig, GsGeometry, GsProfile, check, lib
from .graph import BUCKET_DTYPE, Geometry, _as_pairs, _device_stream, _stream_ptr


def tenant_bytes(num_vertices: int, sketches_factor: float = 1.0) -> int:
    """Device bytes one tenant's sketches take: what admission charges against the budget."""
    out = C.c_uint64()
    check(lib().gs_engine_tenant_bytes(num_vertices, sketches_factor, C.byref(out)), "gs_engine_tenant_bytes")
    return out.value


@dataclass
class TenantResult:
    labels: np.ndarray | None  # smallest tenant-local vertex id of each vertex's component
    num_cc: int
    rounds: int


class SketchEngine:
    """Device arena of tenant sketches with admission by sketch bytes."""

    def __init__(self, sketch_budget_bytes: int, max_tenants: int, max_vertices: int, max_tenant_vertices: int,
                 device: int = -1, max_batch_edges: int = 0):
        self._lib = lib()
        cfg = GsEngineConfig(sketch_budget_bytes, max_tenants, max_vertices, max_tenant_vertices, device,
                             max_batch_edges)
        h = C.c_void_p()
        check(self._lib.gs_engine_create(C.byref(cfg), C.byref(h)), "gs_engine_create")
        self._h = h
        self.tenants: dict[int, int] = {}  # tenant id -> num_vertices

    # ---- lifecycle ----
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.gs_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream=None) -> None:
        check(self._lib.gs_engine_set_stream(self._h, _stream_ptr(stream)), "gs_engine_set_stream")

    # ---- admission ----
    def add_tenant(self, num_vertices: int, seed: int, sketches_factor: float = 1.0) -> int:
        """Tenant id; raises GpuSketchError with status GS_ERR_OOM when it cannot be admitted now."""
        t = C.c_uint32()
        check(self._lib.gs_engine_add_tenant(self._h, num_vertices, seed & (2**64 - 1), sketches_factor, C.byref(t)),
              "gs_engine_add_tenant")
        self.tenants[t.value] = num_vertices
        return t.value

    def try_add_tenant(self, num_vertices: int, seed: int, sketches_factor: float = 1.0) -> int | None:
        """Tenant id, or None when the arena, vertex space or tenant slots are full."""
        try:
            return self.add_tenant(num_vertices, seed, sketches_factor)
        except GpuSketchError as e:
            if e.status == GS_ERR_OOM:
                return None
            raise

    def remove_tenant(self, tenant: int) -> None:
        check(self._lib.gs_engine_remove_tenant(self._h, tenant), "gs_engine_remove_tenant")
        self.tenants.pop(tenant, None)

    def clear_tenant(self, tenant: int) -> None:
        """Zero one tenant's sketches."""
        check(self._lib.gs_engine_clear_tenant(self._h, tenant), "gs_engine_clear_tenant")

    def memory(self) -> tuple[int, int, int]:
        """(sketch bytes in use, arena bytes, live tenants)."""
        u, c, n = C.c_uint64(), C.c_uint64(), C.c_uint32()
        check(self._lib.gs_engine_memory(self._h, C.byref(u), C.byref(c), C.byref(n)), "gs_engine_memory")
        return u.value, c.value, n.value

    def geometry(self, tenant: int) -> Geometry:
        g = GsGeometry()
        check(self._lib.gs_engine_tenant_geometry(self._h, tenant, C.byref(g)), "gs_engine_tenant_geometry")
        return Geometry._from(g)

    # ---- ingest ----
    def ingest(self, slice_tenants, slice_offsets, pairs, stream=None) -> None:
        """Slices of records: slice i is pairs[slice_offsets[i]:slice_offsets[i+1]] of tenant slice_tenants[i]."""
        st = np.ascontiguousarray(slice_tenants, dtype=np.uint32)
        so = np.ascontiguousarray(slice_offsets, dtype=np.uint64)
        if so.size != st.size + 1:
            raise ValueError("slice_offsets needs one entry more than slice_tenants")
        p, _, dev, keep = _as_pairs(pairs)
        check(self._lib.gs_engine_ingest(self._h, st.ctypes.data, so.ctypes.data, st.size, p, int(dev),
                                         _device_stream(stream, dev)), "gs_engine_ingest")
        del keep

    def ingest_batches(self, batches, stream=None) -> None:
        """batches: iterable of (tenant, (n, 2) uint32 host array); concatenated into one ingest call."""
        tens, parts, offs = [], [], [0]
        for t, a in batches:
            a = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, 2)
            tens.append(t)
            parts.append(a)
            offs.append(offs[-1] + a.shape[0])
        if not tens:
            return
        self.ingest(tens, offs, np.concatenate(parts) if len(parts) > 1 else parts[0], stream)

    def ingest_slices(self, batches, stream=None) -> None:
        """batches: iterable of (tenant, (n, 2) uint32 host array or CPU tensor), one coalesced ingest
        without concatenating on the host (page-locked arrays are copied to the device directly)."""
        keep, tens, counts, ptrs = [], [], [], []
        for t, a in batches:
            p, n, dev, k = _as_pairs(a)
            if dev:
                raise ValueError("ingest_slices takes host records")
            keep.append(k)
            tens.append(t)
            counts.append(n)
            ptrs.append(p.value or 0)
        if not tens:
            return
        st = np.array(tens, np.uint32)
        sc = np.array(counts, np.uint64)
        sp = (C.c_void_p * len(ptrs))(*ptrs)
        check(self._lib.gs_engine_ingest_slices(self._h, len(tens), st.ctypes.data, sc.ctypes.data, sp,
                                                _stream_ptr(stream)), "gs_engine_ingest_slices")
        del keep

    def synchronize(self) -> None:
        check(self._lib.gs_engine_synchronize(self._h), "gs_engine_synchronize")

    def phase(self, slice_tenants, slice_offsets, pairs, query_tenants=(), cuda_graph: bool = True) -> dict:
        """One batched phase: ingest device-resident slices, then query `query_tenants` (no labels).
        With cuda_graph the phase's device work runs as one CUDA graph.  {tenant: (num_cc, rounds)}."""
        st = np.ascontiguousarray(slice_tenants, dtype=np.uint32)
        so = np.ascontiguousarray(slice_offsets, dtype=np.uint64)
        if so.size != st.size + 1:
            raise ValueError("slice_offsets needs one entry more than slice_tenants")
        p, _, dev, keep = _as_pairs(pairs)
        if not dev and st.size:
            raise ValueError("phase() takes device-resident records (a CUDA tensor)")
        if dev:
            # gs_engine_phase takes no stream: the records' producer (and a .contiguous() copy) must be
            # complete before the engine's own stream reads them
            import torch
            torch.cuda.current_stream().synchronize()
        qt = np.ascontiguousarray(list(query_tenants), dtype=np.uint32)
        ncc = np.zeros(max(qt.size, 1), np.uint32)
        rounds = np.zeros(max(qt.size, 1), np.uint32)
        check(self._lib.gs_engine_phase(self._h, st.ctypes.data, so.ctypes.data, st.size, p, qt.ctypes.data, qt.size,
                                        ncc.ctypes.data, rounds.ctypes.data,
                                        GS_PHASE_CUDA_GRAPH if cuda_graph else 0), "gs_engine_phase")
        del keep
        return {int(t): (int(ncc[i]), int(rounds[i])) for i, t in enumerate(qt)}

    def graph_stats(self) -> tuple[int, int]:
        """(CUDA graphs instantiated, CUDA graph launches) by phase() so far."""
        b, l = C.c_uint64(), C.c_uint64()
        check(self._lib.gs_engine_graph_stats(self._h, C.byref(b), C.byref(l)), "gs_engine_graph_stats")
        return b.value, l.value

    # ---- queries ----
    def connected_components(self, tenants, with_labels: bool = True) -> dict[int, TenantResult]:
        ts = np.ascontiguousarray(list(tenants), dtype=np.uint32)
        n = ts.size
        if n == 0:
            return {}
        sizes = [self.tenants[int(t)] for t in ts]
        labels = np.empty(sum(sizes), np.uint32) if with_labels else None
        ncc = np.zeros(n, np.uint32)
        rounds = np.zeros(n, np.uint32)
        check(self._lib.gs_engine_connected_components(self._h, ts.ctypes.data, n,
                                                       labels.ctypes.data if with_labels else None,
                                                       ncc.ctypes.data, rounds.ctypes.data),
              "gs_engine_connected_components")
        out, off = {}, 0
        for i, t in enumerate(ts):
            lab = labels[off: off + sizes[i]] if with_labels else None
            out[int(t)] = TenantResult(lab, int(ncc[i]), int(rounds[i]))
            off += sizes[i]
        return out

    # ---- sketch bytes ----
    def download(self, tenant: int, first: int = 0, count: int | None = None) -> np.ndarray:
        g = self.geometry(tenant)
        count = g.num_vertices - first if count is None else count
        out = np.empty((count, g.num_buckets), BUCKET_DTYPE)
        check(self._lib.gs_engine_download_sketches(self._h, tenant, first, count, out.ctypes.data),
              "gs_engine_download_sketches")
        return out

    def write_binary(self, tenant: int, path: str) -> None:
        check(self._lib.gs_engine_write_binary(self._h, tenant, path.encode()), "gs_engine_write_binary")

    # ---- tuning and profiling ----
    def profile_enable(self, on: bool = True) -> None:
        check(self._lib.gs_engine_profile_enable(self._h, int(on)), "gs_engine_profile_enable")

    def profile_read(self) -> dict:
        p = GsProfile()
        check(self._lib.gs_engine_profile_read(self._h, C.byref(p)), "gs_engine_profile_read")
        return {f: getattr(p, f) for f, _ in GsProfile._fields_}
