"""Reference-named host classes over the C ABI.

Mirrors the reference's algorithm interface so code and tests written against CCSketchAlg /
CCGPUSketchAlg / MCGPUSketchAlg read the same here (include/cc_sketch_alg.h:65-261,
include/cc_gpu_sketch_alg.h:8-110, include/mc_sketch_alg.h:73-304, include/return_types.h).
The sketches live on the GPU; worker-thread batches (apply_update_batch) are buffered on the host
and shipped in bulk, as the reference's CudaStream buffers ~540 batches per launch.
"""
from __future__ import annotations

import threading
from enum import IntEnum
from typing import NamedTuple

import numpy as np

from ._native import GS_ERR_SKETCH_FAIL, GpuSketchError
from .graph import GraphSketch, exact_min_cut

__all__ = [
    "CCAlgConfiguration", "UpdateType", "GraphUpdate", "Edge", "QueryCode", "OutOfSamplesException",
    "UpdateLockedException", "ConnectedComponents", "SpanningForest", "MinCut", "CCSketchAlg", "CCGPUSketchAlg",
    "MCGPUSketchAlg",
]


class UpdateType(IntEnum):
    INSERT = 0
    DELETE = 1
    BREAKPOINT = 2


class QueryCode(IntEnum):
    CONNECTIVITY = 0
    KSPANNINGFORESTS = 1
    MINIMUMCUT = 2


class Edge(NamedTuple):
    src: int
    dst: int


class GraphUpdate(NamedTuple):
    edge: Edge
    type: UpdateType = UpdateType.INSERT


class OutOfSamplesException(RuntimeError):
    """Boruvka needed more rounds than the sketch has columns (include/sketch.h:333-344)."""


class UpdateLockedException(RuntimeError):
    """Update while a query runs (include/cc_sketch_alg.h:25-29)."""


class CCAlgConfiguration:
    """Builder of include/cc_alg_configuration.h: sketches_factor, batch_factor, disk_dir."""

    def __init__(self):
        self._sketches_factor = 1.0
        self._batch_factor = 1.0
        self._disk_dir = "."

    def sketches_factor(self, f: float) -> "CCAlgConfiguration":
        self._sketches_factor = f if f > 0 else 1.0  # src/cc_alg_configuration.cpp:9-17
        return self

    def batch_factor(self, f: float) -> "CCAlgConfiguration":
        self._batch_factor = f if f > 0 else 1.0
        return self

    def disk_dir(self, d: str) -> "CCAlgConfiguration":
        self._disk_dir = d
        return self

    def get_sketches_factor(self) -> float:
        return self._sketches_factor

    def get_batch_factor(self) -> float:
        return self._batch_factor

    def get_disk_dir(self) -> str:
        return self._disk_dir

    def __str__(self) -> str:
        return ("Connected Components Algorithm Configuration:\n Sketching algorithm   = CameoSketch\n"
                " Using Eager DSU       = False\n"
                f" Num sketches factor   = {self._sketches_factor}\n Batch size factor     = {self._batch_factor}\n"
                f" On disk data location = {self._disk_dir}")


class ConnectedComponents:
    """include/return_types.h:10-24: parent array flattened to component ids."""

    def __init__(self, labels: np.ndarray):
        self._labels = labels
        self._num_cc = int(np.count_nonzero(labels == np.arange(len(labels), dtype=labels.dtype)))

    def size(self) -> int:
        return self._num_cc

    def is_connected(self, a: int, b: int) -> bool:
        return bool(self._labels[a] == self._labels[b])

    def labels(self) -> np.ndarray:
        return self._labels

    def get_component_sets(self) -> list[set[int]]:
        order = np.argsort(self._labels, kind="stable")
        lab = self._labels[order]
        cuts = np.flatnonzero(np.diff(lab)) + 1
        return [set(map(int, part)) for part in np.split(order, cuts)]


class SpanningForest:
    """include/return_types.h:26-38."""

    def __init__(self, edges: np.ndarray):
        self._edges = np.asarray(edges, dtype=np.uint32).reshape(-1, 2)

    def get_edges(self) -> list[Edge]:
        return [Edge(int(a), int(b)) for a, b in self._edges]

    def edge_array(self) -> np.ndarray:
        return self._edges

    def get_sorted_adjacency(self) -> list[Edge]:
        both = np.concatenate([self._edges, self._edges[:, ::-1]])
        both = both[np.lexsort((both[:, 1], both[:, 0]))]
        return [Edge(int(a), int(b)) for a, b in both]


class MinCut(NamedTuple):
    left_vertices: set
    right_vertices: set
    value: int


def _raise(e: GpuSketchError):
    if e.status == GS_ERR_SKETCH_FAIL:
        raise OutOfSamplesException(str(e)) from e
    raise e


class CCGPUSketchAlg:
    """Connected components over a device-resident sketch set (CCGPUSketchAlg drop-in).

    Constructor arguments follow CCSketchAlg(num_vertices, seed, config); `num_threads` sizes the
    per-worker batch buffers like CCGPUSketchAlg's num_threads (include/cc_gpu_sketch_alg.h:36).
    """

    def __init__(self, num_vertices: int, seed: int, config: CCAlgConfiguration | None = None,
                 num_threads: int = 1, device: int = -1):
        self.config = config or CCAlgConfiguration()
        self._g = GraphSketch(num_vertices, seed, self.config.get_sketches_factor(),
                              self.config.get_batch_factor(), device=device)
        self.num_vertices = num_vertices
        self.seed = seed
        self._lock = threading.Lock()
        self._buf: dict[int, list] = {}
        self._buffered = 0
        self._flush_at = max(1, 540 * self.get_desired_updates_per_batch() // 4)
        self.allocate_worker_memory(num_threads)
        self.last_query_rounds = 0
        self._last_forest = np.empty((0, 2), np.uint32)
        self.update_locked = False

    # driver contract (include/graph_sketch_driver.h:28-69)
    def allocate_worker_memory(self, num_workers: int) -> None:
        self._num_workers = num_workers

    def get_desired_updates_per_batch(self) -> int:
        return int(self._g._lib.gs_desired_updates_per_batch(self._g._h))

    def get_num_vertices(self) -> int:
        return self.num_vertices

    def get_seed(self) -> int:
        return self.seed

    def max_rounds(self) -> int:
        return self._g.geometry.num_samples

    def pre_insert(self, upd: GraphUpdate, thr_id: int = 0) -> None:
        """Nothing to do here: with set_eager_dsu(True) the library keeps its DSU current on every
        ingested edge record (CCSketchAlg::pre_insert, src/cc_sketch_alg.cpp:106-131)."""

    def set_eager_dsu(self, on: bool = True) -> None:
        """Library extension: the eager DSU answers connected_components() without Boruvka while
        no ingested record may have deleted a forest edge (off by default, like NO_EAGER_DSU)."""
        self._g.set_eager_dsu(on)

    def has_cached_query(self, query_code: int) -> bool:
        if query_code != QueryCode.CONNECTIVITY:
            return False
        return self._g.has_cached_query()

    def print_configuration(self) -> None:
        print(self.config)

    def apply_update_batch(self, thr_id: int, src_vertex: int, dst_vertices) -> None:
        """Buffers one worker batch (edges src->dst, applied to src's sketch only)."""
        if self.update_locked:
            raise UpdateLockedException("Cannot update the algorithm: Connected components currently running")
        d = np.asarray(dst_vertices, dtype=np.uint32)
        with self._lock:
            self._buf.setdefault(src_vertex, []).append(d)
            self._buffered += d.size
            if self._buffered >= self._flush_at:
                self._ship_locked()

    def _ship_locked(self) -> None:
        if not self._buf:
            return
        srcs = np.fromiter(self._buf.keys(), np.uint32, len(self._buf))
        parts = [np.concatenate(v) if len(v) > 1 else v[0] for v in self._buf.values()]
        sizes = np.fromiter((p.size for p in parts), np.uint64, len(parts))
        starts = np.zeros_like(sizes)
        np.cumsum(sizes[:-1], out=starts[1:])
        dsts = np.concatenate(parts) if parts else np.empty(0, np.uint32)
        self._g.ingest_vertex_batches(srcs, starts, sizes, dsts)
        self._buf.clear()
        self._buffered = 0

    def flush_buffers(self) -> None:
        """src/cc_gpu_sketch_alg.cpp:21-31."""
        with self._lock:
            self._ship_locked()
        self._g.synchronize()

    def update(self, upd: GraphUpdate) -> None:
        """Direct edge update of both endpoints (src/cc_sketch_alg.cpp:154-160)."""
        e = upd.edge
        self._g.ingest_pairs(np.array([[e[0], e[1]]], np.uint32))

    def ingest_pairs(self, pairs, stream=None) -> None:
        """Bulk edge records (n, 2): the device-bucketed fast path."""
        self._g.ingest_pairs(pairs, stream)

    # queries
    def connected_components(self) -> ConnectedComponents:
        self.flush_buffers()
        try:
            labels, _, rounds = self._g.connected_components(0)
        except GpuSketchError as e:
            _raise(e)
        self.last_query_rounds = rounds
        return ConnectedComponents(labels)

    def point_query(self, a: int, b: int) -> bool:
        self.flush_buffers()
        try:
            return self._g.point_query(a, b)
        except GpuSketchError as e:
            _raise(e)

    def calc_spanning_forest(self) -> SpanningForest:
        self.flush_buffers()
        try:
            return SpanningForest(self._g.spanning_forest(0))
        except GpuSketchError as e:
            _raise(e)

    def calc_disjoint_spanning_forests(self, k: int) -> list[SpanningForest]:
        self.flush_buffers()
        try:
            return [SpanningForest(f) for f in self._g.disjoint_spanning_forests(k, 0)]
        except GpuSketchError as e:
            _raise(e)

    def write_binary(self, filename: str) -> None:
        self.flush_buffers()
        self._g.write_binary(filename)

    @staticmethod
    def construct_from_serialized_data(input_file: str, config: CCAlgConfiguration | None = None) -> "CCGPUSketchAlg":
        g = GraphSketch.read_binary(input_file)
        obj = CCGPUSketchAlg.__new__(CCGPUSketchAlg)
        obj.config = (config or CCAlgConfiguration())
        obj._g = g
        obj.num_vertices = g.num_vertices
        obj.seed = g.seed
        obj._lock = threading.Lock()
        obj._buf = {}
        obj._buffered = 0
        obj._flush_at = max(1, 540 * obj.get_desired_updates_per_batch() // 4)
        obj._num_workers = 1
        obj.last_query_rounds = 0
        obj.update_locked = False
        return obj

    def sketches(self) -> GraphSketch:
        return self._g


# the CPU class name maps to the same device implementation
CCSketchAlg = CCGPUSketchAlg


class MCGPUSketchAlg:
    """k-connectivity / minimum cut over per-level sketch subgraphs (MCGPUSketchAlg drop-in).

    num_subgraphs is the tag bound L of get_index_depth(e, seed, L-1) (src/mc_gpu_sketch_alg.cpp:160);
    max_sketch_graphs levels are kept as sketches.
    """

    def __init__(self, num_vertices: int, seed: int, num_subgraphs: int, max_sketch_graphs: int, k: int,
                 config: CCAlgConfiguration | None = None, device: int = -1):
        self.config = config or CCAlgConfiguration()
        self.k = k
        self.num_vertices = num_vertices
        self.seed = seed
        self._g = GraphSketch(num_vertices, seed, self.config.get_sketches_factor(), self.config.get_batch_factor(),
                              num_levels=max_sketch_graphs, num_subgraphs=num_subgraphs, device=device)

    def get_num_vertices(self) -> int:
        return self.num_vertices

    def get_num_sketch_graphs(self) -> int:
        return self._g.num_levels

    def ingest_pairs(self, pairs, stream=None) -> None:
        self._g.ingest_pairs(pairs, stream)

    def update(self, upd: GraphUpdate) -> None:
        e = upd.edge
        self._g.ingest_pairs(np.array([[e[0], e[1]]], np.uint32))

    def apply_flush_updates(self) -> None:
        self._g.synchronize()

    def calc_disjoint_spanning_forests(self, graph_id: int, k: int) -> list[SpanningForest]:
        try:
            return [SpanningForest(f) for f in self._g.disjoint_spanning_forests(k, graph_id)]
        except GpuSketchError as e:
            _raise(e)

    def calc_minimum_cut(self, edges) -> MinCut:
        e = np.asarray([[a, b] for a, b in edges], np.uint32) if not isinstance(edges, np.ndarray) else edges
        value, side = exact_min_cut(self.num_vertices, e)
        left = set(np.flatnonzero(side).tolist())
        return MinCut(left, set(range(self.num_vertices)) - left, int(value))

    def min_cut(self, k: int | None = None):
        """tools/min_cut.cu:208-252 on the device: (value, level, cut at that level)."""
        try:
            v, lvl, cut, _ = self._g.min_cut(k or self.k)
        except GpuSketchError as e:
            _raise(e)
        return v, lvl, cut

    def sketches(self) -> GraphSketch:
        return self._g
