"""GraphSketch: one device-resident sketch set behind the C ABI (include/gpusketch.h).

Arrays may be numpy arrays (host memory) or torch tensors (host or CUDA memory); CUDA tensors are
passed to the library as device pointers, so the records never leave HBM.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._native import GsGeometry, GsGraphConfig, GsProfile, check, lib

BUCKET_DTYPE = np.dtype([("alpha", "<u8"), ("gamma", "<u8")])


@dataclass(frozen=True)
class Geometry:
    """Sketch sizes derived as the reference's Sketch::calc_* functions do."""
    num_vertices: int
    num_samples: int
    cols_per_sample: int
    num_columns: int
    bkt_per_col: int
    num_buckets: int
    bytes_per_vertex: int

    @staticmethod
    def _from(g: GsGeometry) -> "Geometry":
        return Geometry(g.num_vertices, g.num_samples, g.cols_per_sample, g.num_columns, g.bkt_per_col,
                        g.num_buckets, g.bytes_per_vertex)


def geometry_for(num_vertices: int, sketches_factor: float = 1.0) -> Geometry:
    g = GsGeometry()
    check(lib().gs_geometry_for(num_vertices, sketches_factor, C.byref(g)), "gs_geometry_for")
    return Geometry._from(g)


def hash64(key: int, seed: int) -> int:
    """XXH3_64bits_withSeed of an 8-byte key, as the device computes it."""
    return int(lib().gs_hash64(key & (2**64 - 1), seed & (2**64 - 1)))


def _as_pairs(pairs):
    """(pointer, count, on_device, keepalive) for an (n, 2) uint32 array or tensor."""
    try:
        import torch
        if isinstance(pairs, torch.Tensor):
            if pairs.dtype not in (torch.int32, torch.uint32):
                raise TypeError("edge records must be 32-bit integers")
            t = pairs.contiguous()
            return C.c_void_p(t.data_ptr()), t.numel() // 2, bool(t.is_cuda), t
    except ImportError:  # pragma: no cover
        pass
    a = np.ascontiguousarray(pairs, dtype=np.uint32)
    return C.c_void_p(a.ctypes.data), a.size // 2, False, a


def _as_u32(values):
    """(pointer, count, on_device, keepalive) for a 1-D uint32 array or 32-bit tensor."""
    try:
        import torch
        if isinstance(values, torch.Tensor):
            if values.dtype not in (torch.int32, torch.uint32):
                raise TypeError("vertex ids must be 32-bit integers")
            t = values.contiguous()
            return C.c_void_p(t.data_ptr()), t.numel(), bool(t.is_cuda), t
    except ImportError:  # pragma: no cover
        pass
    a = np.ascontiguousarray(values, dtype=np.uint32)
    return C.c_void_p(a.ctypes.data), a.size, False, a


def _stream_ptr(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(0)
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


def _device_stream(stream, on_device: bool) -> C.c_void_p:
    """The stream a call with device operands runs on.  With no explicit stream, torch's current
    stream: the library's work is then ordered after the torch kernels that produced the operands, and
    torch's caching allocator, which reuses a freed block only after the work queued on that stream,
    cannot hand a temporary (a .contiguous() copy) to another tensor while the library still reads it."""
    if stream is None and on_device:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _stream_ptr(stream)


class GraphSketch:
    """A sketch set of `num_levels` levels of V vertex sketches resident on one GPU."""

    def __init__(self, num_vertices: int, seed: int, sketches_factor: float = 1.0, batch_factor: float = 1.0,
                 num_levels: int = 1, num_subgraphs: int = 0, device: int = -1, max_batch_edges: int = 0,
                 _handle: C.c_void_p | None = None):
        self._lib = lib()
        if _handle is not None:
            self._h = _handle
        else:
            cfg = GsGraphConfig(num_vertices, num_levels, seed & (2**64 - 1), sketches_factor, batch_factor,
                                num_subgraphs, device, max_batch_edges)
            h = C.c_void_p()
            check(self._lib.gs_graph_create(C.byref(cfg), C.byref(h)), "gs_graph_create")
            self._h = h
        g = GsGeometry()
        check(self._lib.gs_graph_geometry(self._h, C.byref(g)), "gs_graph_geometry")
        self.geometry = Geometry._from(g)
        self.num_vertices = self.geometry.num_vertices
        self.num_levels = num_levels if _handle is None else 1
        self.seed = seed

    # ---- lifecycle ----
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.gs_graph_destroy(self._h)
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

    def clear(self) -> None:
        """Zero every sketch (Sketch::zero_contents over the set)."""
        check(self._lib.gs_clear(self._h), "gs_clear")

    def set_stream(self, stream=None) -> None:
        """Launch this handle's kernels on `stream` (a torch.cuda.Stream or cudaStream_t int); None = own."""
        check(self._lib.gs_graph_set_stream(self._h, _stream_ptr(stream)), "gs_graph_set_stream")

    # ---- ingest ----
    def ingest_pairs(self, pairs, stream=None) -> None:
        p, n, dev, keep = _as_pairs(pairs)
        check(self._lib.gs_ingest_pairs(self._h, p, n, int(dev), _device_stream(stream, dev)), "gs_ingest_pairs")
        del keep

    def prepare_host_input(self, records: int) -> None:
        """gs_prepare_host_input: allocate the page-locked staging ring for host slices of `records` now."""
        check(self._lib.gs_prepare_host_input(self._h, records), "gs_prepare_host_input")

    def ingest_pairs_async(self, pairs, stream=None) -> None:
        """gs_ingest_pairs_async: queue the copies and the ingest without waiting.  A page-locked host
        buffer (a pinned CPU tensor) stays in use until the handle's queued work is done: keep it alive
        and unchanged until synchronize(), query_wait() or a synchronous query."""
        p, n, dev, keep = _as_pairs(pairs)
        if keep is not pairs and not dev:
            raise ValueError("ingest_pairs_async needs a C-contiguous uint32/int32 buffer the caller keeps alive")
        check(self._lib.gs_ingest_pairs_async(self._h, p, n, int(dev), _device_stream(stream, dev)),
              "gs_ingest_pairs_async")

    def ingest_stream_file(self, path: str, first: int = 0, count: int | None = None) -> int:
        """gs_ingest_stream_file: records [first, first+count) of a binary stream file; returns the number
        of records ingested."""
        n = C.c_uint64()
        check(self._lib.gs_ingest_stream_file(self._h, str(path).encode(), first,
                                              2**64 - 1 if count is None else count, C.byref(n)),
              "gs_ingest_stream_file")
        return n.value

    def ingest_edges(self, src, dst, stream=None) -> None:
        """gs_ingest_edges: record i toggles edge {src[i], dst[i]}; both arrays on the host or both on
        the device."""
        a, na, da, ka = _as_u32(src)
        b, nb, db, kb = _as_u32(dst)
        if na != nb or da != db:
            raise ValueError("src and dst need the same length and the same side (host or device)")
        check(self._lib.gs_ingest_edges(self._h, a, b, na, int(da), _device_stream(stream, da)), "gs_ingest_edges")
        del ka, kb

    def ingest_vertex_batches(self, srcs, starts, sizes, dsts, level: int = 0) -> None:
        s = np.ascontiguousarray(srcs, dtype=np.uint32)
        st = np.ascontiguousarray(starts, dtype=np.uint64)
        sz = np.ascontiguousarray(sizes, dtype=np.uint64)
        d = np.ascontiguousarray(dsts, dtype=np.uint32)
        check(self._lib.gs_ingest_vertex_batches(self._h, level, s.ctypes.data, st.ctypes.data, sz.ctypes.data,
                                                 len(s), d.ctypes.data, d.size, 0, None),
              "gs_ingest_vertex_batches")

    def synchronize(self) -> None:
        check(self._lib.gs_synchronize(self._h), "gs_synchronize")

    # ---- queries ----
    def connected_components(self, level: int = 0):
        """(labels, num_cc, rounds); labels[v] = smallest vertex id in v's component."""
        labels = np.empty(self.num_vertices, np.uint32)
        ncc, rounds = C.c_uint32(), C.c_uint32()
        check(self._lib.gs_connected_components(self._h, level, labels.ctypes.data, C.byref(ncc), C.byref(rounds)),
              "gs_connected_components")
        return labels, ncc.value, rounds.value

    def connected_components_async(self, level: int = 0) -> None:
        """Queue connected_components(level); collect the answer with query_wait()."""
        check(self._lib.gs_connected_components_async(self._h, level), "gs_connected_components_async")

    def query_wait(self):
        """(labels, num_cc, rounds) of the query queued by connected_components_async()."""
        labels = np.empty(self.num_vertices, np.uint32)
        ncc, rounds = C.c_uint32(), C.c_uint32()
        check(self._lib.gs_query_wait(self._h, labels.ctypes.data, C.byref(ncc), C.byref(rounds)), "gs_query_wait")
        return labels, ncc.value, rounds.value

    def point_query(self, a: int, b: int) -> bool:
        out = C.c_int()
        check(self._lib.gs_point_query(self._h, a, b, C.byref(out)), "gs_point_query")
        return bool(out.value)

    def spanning_forest(self, level: int = 0) -> np.ndarray:
        edges = np.empty(2 * self.num_vertices, np.uint32)
        n = C.c_uint64()
        check(self._lib.gs_spanning_forest(self._h, level, edges.ctypes.data, C.byref(n)), "gs_spanning_forest")
        return edges[: 2 * n.value].reshape(-1, 2).copy()

    def disjoint_spanning_forests(self, k: int, level: int = 0) -> list[np.ndarray]:
        stride = 2 * (self.num_vertices - 1)
        edges = np.zeros(k * stride, np.uint32)
        sizes = np.zeros(k, np.uint64)
        check(self._lib.gs_disjoint_spanning_forests(self._h, level, k, edges.ctypes.data, sizes.ctypes.data),
              "gs_disjoint_spanning_forests")
        return [edges[f * stride: f * stride + 2 * int(sizes[f])].reshape(-1, 2).copy() for f in range(k)]

    def min_cut(self, k: int):
        """(value, level, cut_at_level, side) of the level-by-level k-forest certificate driver."""
        value, lvl, cut = C.c_uint64(), C.c_uint32(), C.c_uint64()
        side = np.zeros(self.num_vertices, np.uint8)
        check(self._lib.gs_min_cut(self._h, k, C.byref(value), C.byref(lvl), C.byref(cut), side.ctypes.data),
              "gs_min_cut")
        return value.value, lvl.value, cut.value, side

    def set_edge_store(self, initial_sketch_levels: int, store_bytes: int = 0) -> None:
        """gs_graph_set_edge_store: start with `initial_sketch_levels` sketched levels and turn the exact
        tier's lowest level into a sketch level whenever it holds store_bytes / 16 edges."""
        check(self._lib.gs_graph_set_edge_store(self._h, initial_sketch_levels, store_bytes), "gs_graph_set_edge_store")

    def sketched_levels(self) -> tuple[int, int]:
        """(levels sketched now, contractions so far)."""
        lv, c = C.c_uint32(), C.c_uint64()
        check(self._lib.gs_graph_sketched_levels(self._h, C.byref(lv), C.byref(c)), "gs_graph_sketched_levels")
        return lv.value, c.value

    def edge_store_edges(self, min_tag: int | None = None) -> np.ndarray:
        """Present edges of the exact tier with subgraph tag >= min_tag (default: the sketched levels)."""
        t = self.sketched_levels()[0] if min_tag is None else min_tag
        n = C.c_uint64()
        check(self._lib.gs_edge_store_edges(self._h, t, None, 0, C.byref(n)), "gs_edge_store_edges")
        out = np.empty((max(n.value, 1), 2), np.uint32)
        check(self._lib.gs_edge_store_edges(self._h, t, out.ctypes.data, n.value, C.byref(n)), "gs_edge_store_edges")
        return out[: n.value].copy()

    def set_device_wait_limit(self, nanoseconds: int = 0) -> None:
        """Limit of the Boruvka kernel's grid-barrier waits (0 = the default, about a second)."""
        check(self._lib.gs_set_device_wait_limit(self._h, nanoseconds), "gs_set_device_wait_limit")

    # ---- eager DSU ----
    def set_eager_dsu(self, on: bool = True) -> None:
        """Keep a device DSU current during ingest so that queries skip Boruvka while it is valid."""
        check(self._lib.gs_set_eager_dsu(self._h, int(on)), "gs_set_eager_dsu")

    def has_cached_query(self) -> bool:
        out = C.c_int()
        check(self._lib.gs_has_cached_query(self._h, C.byref(out)), "gs_has_cached_query")
        return bool(out.value)

    # ---- profiling ----
    def profile_enable(self, on: bool = True) -> None:
        check(self._lib.gs_profile_enable(self._h, int(on)), "gs_profile_enable")

    def profile_read(self) -> dict:
        p = GsProfile()
        check(self._lib.gs_profile_read(self._h, C.byref(p)), "gs_profile_read")
        return {f: getattr(p, f) for f, _ in GsProfile._fields_}

    # ---- sketch bytes ----
    def download(self, level: int = 0, first: int = 0, count: int | None = None) -> np.ndarray:
        count = self.num_vertices - first if count is None else count
        out = np.empty((count, self.geometry.num_buckets), BUCKET_DTYPE)
        check(self._lib.gs_download_sketches(self._h, level, first, count, out.ctypes.data), "gs_download_sketches")
        return out

    def upload(self, buckets: np.ndarray, level: int = 0, first: int = 0) -> None:
        b = np.ascontiguousarray(buckets, dtype=BUCKET_DTYPE).reshape(-1, self.geometry.num_buckets)
        check(self._lib.gs_upload_sketches(self._h, level, first, b.shape[0], b.ctypes.data), "gs_upload_sketches")

    def write_binary(self, path: str) -> None:
        check(self._lib.gs_write_binary(self._h, path.encode()), "gs_write_binary")

    @staticmethod
    def read_binary(path: str, device: int = -1) -> "GraphSketch":
        h = C.c_void_p()
        check(lib().gs_read_binary(path.encode(), device, C.byref(h)), "gs_read_binary")
        with open(path, "rb") as f:
            seed = int.from_bytes(f.read(8), "little")
        return GraphSketch(0, seed, _handle=h)


def exact_min_cut(num_vertices: int, edges) -> tuple[int, np.ndarray]:
    """Exact global minimum cut of a multigraph (host C++ in the library)."""
    e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1)
    v = C.c_uint64()
    side = np.zeros(num_vertices, np.uint8)
    check(lib().gs_exact_min_cut(num_vertices, e.ctypes.data, e.size // 2, C.byref(v), side.ctypes.data),
          "gs_exact_min_cut")
    return v.value, side


def er_stream(num_vertices: int, p: float, seed: int, delete_frac: float = 0.0, reinsert_frac: float = 0.0) -> np.ndarray:
    """Seeded Erdos-Renyi dynamic stream as an (n, 2) uint32 array (host generator in the library)."""
    n = C.c_uint64()
    check(lib().gs_gen_er_stream(num_vertices, p, seed, delete_frac, reinsert_frac, None, 0, C.byref(n)),
          "gs_gen_er_stream")
    out = np.empty((n.value, 2), np.uint32)
    check(lib().gs_gen_er_stream(num_vertices, p, seed, delete_frac, reinsert_frac, out.ctypes.data, n.value,
                                 C.byref(n)), "gs_gen_er_stream")
    return out


def rmat_stream(log2_v: int, n: int, seed: int, first: int = 0, a: float = 0.57, b: float = 0.19, c: float = 0.19,
                delete_frac: float = 0.12, out=None, stream=None):
    """Counter-based R-MAT records [first, first+n).  `out` may be a CUDA tensor (generated on the device)."""
    if out is None:
        out = np.empty((n, 2), np.uint32)
    p, cnt, dev, keep = _as_pairs(out)
    if cnt < n:
        raise ValueError("output too small")
    check(lib().gs_gen_rmat_stream(log2_v, a, b, c, delete_frac, seed, first, n, p, int(dev),
                                   _device_stream(stream, dev)), "gs_gen_rmat_stream")
    return out
