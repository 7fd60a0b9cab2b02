"""ctypes bindings of the oracle libraries (TEST INFRASTRUCTURE ONLY; see oracle/__init__.py)."""
from __future__ import annotations

import ctypes as C
import os
import struct
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libgsoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgsref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libgsrefgpu.so")

_u32 = np.ctypeslib.ndpointer(np.uint32, flags="C")
_u64 = np.ctypeslib.ndpointer(np.uint64, flags="C")
_u8 = np.ctypeslib.ndpointer(np.uint8, flags="C")

GOOD, ZERO, FAIL = 0, 1, 2


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise RuntimeError(f"{path} missing: run `make -f oracle/Makefile`")
    return C.CDLL(path)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class Restatement:
    """The plain-C restatement (oracle/gsoracle.c)."""

    def __init__(self):
        L = _load(ORACLE_SO)
        L.or_xxh3_8.restype = C.c_uint64
        L.or_xxh3_8.argtypes = [C.c_uint64, C.c_uint64]
        L.or_index_depth.restype = C.c_uint32
        L.or_index_depth.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32]
        L.or_geometry.argtypes = [C.c_uint32, C.c_double, _u32]
        L.or_ingest_pairs.argtypes = [_u64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, _u32, C.c_uint64]
        L.or_ingest_pairs_levels.argtypes = [_u64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                             C.c_uint32, C.c_uint64, _u32, C.c_uint64]
        L.or_sketch_update.argtypes = [_u64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64]
        L.or_sample.restype = C.c_int
        L.or_sample.argtypes = [_u64, _u64, C.c_uint32, C.c_uint64, C.POINTER(C.c_uint64)]
        L.or_boruvka.restype = C.c_int
        L.or_boruvka.argtypes = [_u64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, _u32,
                                 C.POINTER(C.c_uint32), _u32, C.POINTER(C.c_uint64)]
        L.or_k_forests.restype = C.c_int
        L.or_k_forests.argtypes = [_u64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                   C.c_uint32, C.c_uint32, _u32, _u64]
        L.or_final_edges.restype = C.c_uint64
        L.or_final_edges.argtypes = [C.c_uint32, _u32, C.c_uint64, _u32]
        L.or_cc_of_edges.restype = C.c_uint32
        L.or_cc_of_edges.argtypes = [C.c_uint32, _u32, C.c_uint64, _u32]
        L.or_stoer_wagner.restype = C.c_uint64
        L.or_stoer_wagner.argtypes = [C.c_uint32, _u32, C.c_uint64, _u8]
        self.L = L

    def xxh3(self, key: int, seed: int) -> int:
        return int(self.L.or_xxh3_8(key & (2**64 - 1), seed & (2**64 - 1)))

    def depth(self, e: int, seed_and_col: int, max_depth: int) -> int:
        return int(self.L.or_index_depth(e, seed_and_col & (2**64 - 1), max_depth))

    def geometry(self, V: int, factor: float = 1.0) -> dict:
        g = np.zeros(5, np.uint32)
        self.L.or_geometry(V, factor, g)
        return dict(num_samples=int(g[0]), cols_per_sample=int(g[1]), num_columns=int(g[2]),
                    bkt_per_col=int(g[3]), num_buckets=int(g[4]))

    def new_sketches(self, V: int, factor: float = 1.0, levels: int = 1) -> np.ndarray:
        g = self.geometry(V, factor)
        return np.zeros(levels * V * g["num_buckets"] * 2, np.uint64)

    def ingest(self, sk: np.ndarray, V: int, seed: int, pairs: np.ndarray, factor: float = 1.0) -> None:
        g = self.geometry(V, factor)
        p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1)
        self.L.or_ingest_pairs(sk, V, g["num_columns"], g["bkt_per_col"], g["num_buckets"], seed, p, p.size // 2)

    def ingest_levels(self, sk: np.ndarray, V: int, levels: int, L: int, seed: int, pairs: np.ndarray,
                      factor: float = 1.0) -> None:
        g = self.geometry(V, factor)
        p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1)
        self.L.or_ingest_pairs_levels(sk, V, levels, L, g["num_columns"], g["bkt_per_col"], g["num_buckets"], seed,
                                      p, p.size // 2)

    def sketch_update(self, one_sketch: np.ndarray, V: int, seed: int, e: int, factor: float = 1.0) -> None:
        g = self.geometry(V, factor)
        self.L.or_sketch_update(one_sketch, g["num_columns"], g["bkt_per_col"], g["num_buckets"], seed, e)

    def boruvka(self, sk: np.ndarray, V: int, seed: int, factor: float = 1.0, round0_col: int = 0):
        """(status, labels, rounds, forest) ; status -1 = out of samples."""
        g = self.geometry(V, factor)
        labels = np.zeros(V, np.uint32)
        forest = np.zeros(2 * V, np.uint32)
        rounds, nf = C.c_uint32(), C.c_uint64()
        st = self.L.or_boruvka(sk, V, g["num_samples"], g["bkt_per_col"], g["num_buckets"], seed, round0_col, labels,
                               C.byref(rounds), forest, C.byref(nf))
        return st, labels, rounds.value, forest[: 2 * nf.value].reshape(-1, 2).copy()

    def k_forests(self, sk_level: np.ndarray, V: int, seed: int, k: int, first_col: int = 0, factor: float = 1.0):
        g = self.geometry(V, factor)
        stride = 2 * (V - 1)
        f = np.zeros(k * stride, np.uint32)
        sizes = np.zeros(k, np.uint64)
        st = self.L.or_k_forests(sk_level, V, g["num_samples"], g["num_columns"], g["bkt_per_col"], g["num_buckets"],
                                 seed, k, first_col, f, sizes)
        return st, [f[j * stride: j * stride + 2 * int(sizes[j])].reshape(-1, 2).copy() for j in range(k)]

    def final_edges(self, V: int, pairs: np.ndarray) -> np.ndarray:
        p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1)
        out = np.zeros(max(2, p.size), np.uint32)
        m = self.L.or_final_edges(V, p, p.size // 2, out)
        return out[: 2 * m].reshape(-1, 2).copy()

    def cc_of_edges(self, V: int, edges: np.ndarray):
        e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1)
        labels = np.zeros(V, np.uint32)
        n = self.L.or_cc_of_edges(V, e, e.size // 2, labels)
        return int(n), labels

    def exact_cc(self, V: int, pairs: np.ndarray):
        return self.cc_of_edges(V, self.final_edges(V, pairs))

    def stoer_wagner(self, V: int, edges: np.ndarray):
        e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1)
        side = np.zeros(V, np.uint8)
        v = self.L.or_stoer_wagner(V, e, e.size // 2, side)
        return int(v), side


def _bind_ref() -> C.CDLL:
    L = _load(REF_SO)
    L.gsref_last_error.restype = C.c_char_p
    L.gsref_cc_new.restype = C.c_void_p
    L.gsref_cc_new.argtypes = [C.c_uint32, C.c_uint64, C.c_double]
    L.gsref_cc_free.argtypes = [C.c_void_p]
    L.gsref_cc_alloc_workers.argtypes = [C.c_void_p, C.c_uint32]
    L.gsref_cc_desired_batch.restype = C.c_uint64
    L.gsref_cc_desired_batch.argtypes = [C.c_void_p]
    L.gsref_cc_update.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_int]
    L.gsref_cc_ingest_batches.argtypes = [C.c_void_p, C.c_uint32, C.c_uint64, _u32, _u64, _u64, _u32]
    L.gsref_cc_connected_components.argtypes = [C.c_void_p, _u32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.gsref_cc_spanning_forest.argtypes = [C.c_void_p, _u32, C.POINTER(C.c_uint64)]
    L.gsref_cc_write_binary.argtypes = [C.c_void_p, C.c_char_p]
    L.gsref_cc_sketch_bytes.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, _u8]
    L.gsref_mc_ingest_tagged.argtypes = [C.c_void_p, _u32, C.c_uint64, C.c_uint32, C.c_uint32]
    L.gsref_mc_level_bytes.argtypes = [C.c_void_p, C.c_uint32, _u8]
    L.gsref_cc_from_file.restype = C.c_void_p
    L.gsref_cc_from_file.argtypes = [C.c_char_p]
    L.gsref_mc_new.restype = C.c_void_p
    L.gsref_mc_new.argtypes = [C.c_uint32, C.c_uint64, C.c_uint32, C.c_double]
    L.gsref_mc_free.argtypes = [C.c_void_p]
    L.gsref_mc_update.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32]
    L.gsref_mc_k_forests.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, _u32, _u64]
    L.gsref_mc_min_cut.restype = C.c_uint64
    L.gsref_mc_min_cut.argtypes = [C.c_void_p, _u32, C.c_uint64, _u8]
    return L


def bucket_by_vertex(pairs: np.ndarray, V: int, batch: int):
    """Both directions of every record grouped by source vertex and cut into batches of at most
    `batch` destinations, as the reference's gutters hand them to apply_update_batch."""
    p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1, 2)
    src = np.concatenate([p[:, 0], p[:, 1]])
    dst = np.concatenate([p[:, 1], p[:, 0]])
    order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order]
    counts = np.bincount(src, minlength=V).astype(np.uint64)
    offs = np.zeros(V + 1, np.uint64)
    np.cumsum(counts, out=offs[1:])
    srcs, starts, sizes = [], [], []
    for v in np.flatnonzero(counts):
        b, e = int(offs[v]), int(offs[v + 1])
        for s in range(b, e, batch):
            srcs.append(v)
            starts.append(s)
            sizes.append(min(batch, e - s))
    return (np.asarray(srcs, np.uint32), np.asarray(starts, np.uint64), np.asarray(sizes, np.uint64),
            np.ascontiguousarray(dst, dtype=np.uint32))


class RefCC:
    """The reference's own CCSketchAlg (NO_EAGER_DSU build)."""

    def __init__(self, V: int, seed: int, factor: float = 1.0, workers: int = 1):
        self.L = _bind_ref()
        self.V = V
        self.h = self.L.gsref_cc_new(V, seed & (2**64 - 1), factor)
        self.L.gsref_cc_alloc_workers(self.h, workers)
        self.workers = workers

    def close(self):
        if self.h:
            self.L.gsref_cc_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update(self, src: int, dst: int, typ: int = 0):
        if self.L.gsref_cc_update(self.h, src, dst, typ):
            raise RuntimeError(self.L.gsref_last_error().decode())

    def ingest(self, pairs: np.ndarray, threads: int | None = None, batch: int | None = None):
        threads = threads or self.workers
        batch = batch or int(self.L.gsref_cc_desired_batch(self.h))
        srcs, starts, sizes, dsts = bucket_by_vertex(pairs, self.V, batch)
        self.ingest_batches(srcs, starts, sizes, dsts, threads)

    def ingest_batches(self, srcs, starts, sizes, dsts, threads: int):
        if self.L.gsref_cc_ingest_batches(self.h, threads, len(srcs), srcs, starts, sizes, dsts):
            raise RuntimeError(self.L.gsref_last_error().decode())

    def connected_components(self):
        labels = np.zeros(self.V, np.uint32)
        ncc, rounds = C.c_uint32(), C.c_uint32()
        rc = self.L.gsref_cc_connected_components(self.h, labels, C.byref(ncc), C.byref(rounds))
        if rc == 2:
            return "out_of_samples", None, None
        if rc:
            raise RuntimeError(self.L.gsref_last_error().decode())
        return labels, ncc.value, rounds.value

    def spanning_forest(self) -> np.ndarray:
        out = np.zeros(2 * self.V, np.uint32)
        n = C.c_uint64()
        if self.L.gsref_cc_spanning_forest(self.h, out, C.byref(n)):
            raise RuntimeError(self.L.gsref_last_error().decode())
        return out[: 2 * n.value].reshape(-1, 2).copy()

    def write_binary_bytes(self) -> bytes:
        with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
            path = f.name
        try:
            self.L.gsref_cc_write_binary(self.h, path.encode())
            with open(path, "rb") as f:
                return f.read()
        finally:
            os.unlink(path)

    def sketch_bytes(self) -> bytes:
        return self.write_binary_bytes()[20:]

    def sketch_array(self, num_buckets: int, first: int = 0, count: int | None = None) -> np.ndarray:
        """The reference Sketch objects' bucket arrays of vertices [first, first+count) as
        (count, num_buckets * 2) uint64, read from memory (no file)."""
        count = self.V - first if count is None else count
        out = np.empty((count, num_buckets * 2), np.uint64)
        self.L.gsref_cc_sketch_bytes(self.h, first, count, out.view(np.uint8).reshape(-1))
        return out


class RefMC:
    """The reference's own MCSketchAlg with `num_graphs` host sketch subgraphs."""

    def __init__(self, V: int, seed: int, num_graphs: int, factor: float = 1.0):
        self.L = _bind_ref()
        self.V = V
        self.num_graphs = num_graphs
        self.h = self.L.gsref_mc_new(V, seed & (2**64 - 1), num_graphs, factor)

    def ingest_tagged(self, pairs: np.ndarray, num_subgraphs: int) -> None:
        """Every record into sketch graphs 0..min(tag, num_graphs-1), tag = the reference's
        get_index_depth(edge id, seed, num_subgraphs-1), through MCSketchAlg::update_subgraph."""
        p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1)
        self.L.gsref_mc_ingest_tagged(self.h, p, p.size // 2, num_subgraphs, self.num_graphs)

    def level_bytes(self, graph_id: int, num_buckets: int) -> bytes:
        out = np.empty(self.V * num_buckets * 16, np.uint8)
        self.L.gsref_mc_level_bytes(self.h, graph_id, out)
        return out.tobytes()

    def close(self):
        if self.h:
            self.L.gsref_mc_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update(self, graph_id: int, src: int, dst: int):
        self.L.gsref_mc_update(self.h, graph_id, src, dst)

    def k_forests(self, graph_id: int, k: int):
        stride = 2 * (self.V - 1)
        f = np.zeros(k * stride, np.uint32)
        sizes = np.zeros(k, np.uint64)
        rc = self.L.gsref_mc_k_forests(self.h, graph_id, k, f, sizes)
        return rc, [f[j * stride: j * stride + 2 * int(sizes[j])].reshape(-1, 2).copy() for j in range(k)]

    def min_cut(self, edges: np.ndarray):
        e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1)
        side = np.zeros(self.V, np.uint8)
        v = self.L.gsref_mc_min_cut(self.h, e, e.size // 2, side)
        return int(v), side


def parse_header(binary: bytes):
    seed, V, factor = struct.unpack_from("<QId", binary, 0)
    return seed, V, factor


def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


class RefGpuKernel:
    """The reference's own GPU sketch-update kernel (src/cuda_kernel.cu:152-257 of the reference, built
    for sm_100a into oracle/_ref/libgsrefgpu.so by oracle/Makefile).  Device pointers are plain ints."""

    def __init__(self):
        L = _load(REF_GPU_SO)
        L.gsref_gpu_prepare.restype = C.c_int
        L.gsref_gpu_prepare.argtypes = [C.c_uint64]
        L.gsref_gpu_sketch_update.restype = C.c_int
        L.gsref_gpu_sketch_update.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                              C.c_uint64, C.c_void_p]
        self.L = L

    def prepare(self, num_buckets: int) -> None:
        assert self.L.gsref_gpu_prepare(num_buckets) == 0

    def sketch_update(self, num_threads, num_batches, stream, d_dsts, d_src, d_sizes, d_start, geo, seed, d_deltas):
        rc = self.L.gsref_gpu_sketch_update(num_threads, num_batches, stream, d_dsts, d_src, d_sizes, d_start,
                                            geo["num_samples"], geo["num_buckets"], geo["num_columns"],
                                            geo["bkt_per_col"], seed, d_deltas)
        assert rc == 0, rc


def ref_batches(pairs: np.ndarray, batch_size: int):
    """The reference's per-vertex batch form of an edge-record stream (GraphSketchDriver gutters ->
    apply_update_batch): both directions of every non-self-loop record, grouped by source vertex,
    each vertex's destinations cut into batches of at most batch_size.  Returns
    (dsts u32, batch src u32, batch start u64, batch size u64)."""
    p = np.asarray(pairs, np.uint32).reshape(-1, 2)
    p = p[p[:, 0] != p[:, 1]]
    src = np.concatenate([p[:, 0], p[:, 1]])
    dst = np.concatenate([p[:, 1], p[:, 0]])
    order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order]
    uniq, first, counts = np.unique(src, return_index=True, return_counts=True)
    nb = (counts + batch_size - 1) // batch_size
    j = np.arange(int(nb.sum())) - np.repeat(np.cumsum(nb) - nb, nb)
    bsrc = np.repeat(uniq, nb).astype(np.uint32)
    bstart = (np.repeat(first, nb) + j * batch_size).astype(np.uint64)
    bsize = np.minimum(batch_size, np.repeat(counts, nb) - j * batch_size).astype(np.uint64)
    return np.ascontiguousarray(dst, np.uint32), bsrc, bstart, bsize
