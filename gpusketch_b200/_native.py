"""ctypes binding of the C ABI in include/gpusketch.h.

The shared library is built in-tree by ``python -m gpusketch_b200.build``.  Loading fails loudly
when it is missing: there is no CPU fallback for any operation of this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpusketch_b200.so")

GS_OK = 0
GS_ERR_BAD_ARG = 1
GS_ERR_CUDA = 2
GS_ERR_OOM = 3
GS_ERR_SKETCH_FAIL = 4
GS_ERR_TIMEOUT = 5
GS_ERR_UPDATE_LOCKED = 6
GS_ERR_IO = 7
GS_ERR_INTERNAL = 8
GS_ERR_NO_DEVICE = 9
GS_PHASE_CUDA_GRAPH = 1

STATUS_NAMES = {
    0: "GS_OK", 1: "GS_ERR_BAD_ARG", 2: "GS_ERR_CUDA", 3: "GS_ERR_OOM", 4: "GS_ERR_SKETCH_FAIL",
    5: "GS_ERR_TIMEOUT", 6: "GS_ERR_UPDATE_LOCKED", 7: "GS_ERR_IO", 8: "GS_ERR_INTERNAL",
    9: "GS_ERR_NO_DEVICE",
}

# every function the header declares: name -> (restype, argtypes)
_P = C.c_void_p
_U32P = C.POINTER(C.c_uint32)
_U64P = C.POINTER(C.c_uint64)
_U8P = C.POINTER(C.c_uint8)


class GsGeometry(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("num_samples", C.c_uint32), ("cols_per_sample", C.c_uint32),
                ("num_columns", C.c_uint32), ("bkt_per_col", C.c_uint32), ("num_buckets", C.c_uint32),
                ("bytes_per_vertex", C.c_uint64)]


class GsGraphConfig(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("num_levels", C.c_uint32), ("seed", C.c_uint64),
                ("sketches_factor", C.c_double), ("batch_factor", C.c_double), ("num_subgraphs", C.c_uint32),
                ("device", C.c_int32), ("max_batch_edges", C.c_uint64)]


class GsProfile(C.Structure):
    _fields_ = [("ingest_launches", C.c_uint64), ("ingest_ms", C.c_double), ("bucket_launches", C.c_uint64),
                ("bucket_ms", C.c_double), ("query_launches", C.c_uint64), ("query_ms", C.c_double),
                ("kernel_launches", C.c_uint64), ("records_ingested", C.c_uint64)]


class GsEngineConfig(C.Structure):
    _fields_ = [("sketch_budget_bytes", C.c_uint64), ("max_tenants", C.c_uint32), ("max_vertices", C.c_uint32),
                ("max_tenant_vertices", C.c_uint32), ("device", C.c_int32), ("max_batch_edges", C.c_uint64)]


SIGNATURES = {
    "gs_geometry_for": (C.c_int, [C.c_uint32, C.c_double, C.POINTER(GsGeometry)]),
    "gs_hash64": (C.c_uint64, [C.c_uint64, C.c_uint64]),
    "gs_graph_create": (C.c_int, [C.POINTER(GsGraphConfig), C.POINTER(_P)]),
    "gs_graph_destroy": (C.c_int, [_P]),
    "gs_graph_geometry": (C.c_int, [_P, C.POINTER(GsGeometry)]),
    "gs_desired_updates_per_batch": (C.c_uint64, [_P]),
    "gs_clear": (C.c_int, [_P]),
    "gs_graph_set_stream": (C.c_int, [_P, _P]),
    "gs_ingest_pairs": (C.c_int, [_P, _P, C.c_uint64, C.c_int, _P]),
    "gs_ingest_edges": (C.c_int, [_P, _P, _P, C.c_uint64, C.c_int, _P]),
    "gs_ingest_pairs_async": (C.c_int, [_P, _P, C.c_uint64, C.c_int, _P]),
    "gs_prepare_host_input": (C.c_int, [_P, C.c_uint64]),
    "gs_ingest_stream_file": (C.c_int, [_P, C.c_char_p, C.c_uint64, C.c_uint64, _U64P]),
    "gs_connected_components_async": (C.c_int, [_P, C.c_uint32]),
    "gs_query_wait": (C.c_int, [_P, _P, _U32P, _U32P]),
    "gs_ingest_vertex_batches": (C.c_int, [_P, C.c_uint32, _P, _P, _P, C.c_uint32, _P, C.c_uint64, C.c_int, _P]),
    "gs_synchronize": (C.c_int, [_P]),
    "gs_graph_set_edge_store": (C.c_int, [_P, C.c_uint32, C.c_uint64]),
    "gs_graph_sketched_levels": (C.c_int, [_P, _U32P, _U64P]),
    "gs_set_device_wait_limit": (C.c_int, [_P, C.c_uint64]),
    "gs_connected_components": (C.c_int, [_P, C.c_uint32, _P, _U32P, _U32P]),
    "gs_point_query": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(C.c_int)]),
    "gs_spanning_forest": (C.c_int, [_P, C.c_uint32, _P, _U64P]),
    "gs_disjoint_spanning_forests": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P]),
    "gs_min_cut": (C.c_int, [_P, C.c_uint32, _U64P, _U32P, _U64P, _P]),
    "gs_exact_min_cut": (C.c_int, [C.c_uint32, _P, C.c_uint64, _U64P, _P]),
    "gs_edge_store_edges": (C.c_int, [_P, C.c_uint32, _P, C.c_uint64, _U64P]),
    "gs_download_sketches": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, _P]),
    "gs_upload_sketches": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, _P]),
    "gs_write_binary": (C.c_int, [_P, C.c_char_p]),
    "gs_read_binary": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(_P)]),
    "gs_set_eager_dsu": (C.c_int, [_P, C.c_int]),
    "gs_has_cached_query": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "gs_get_tuning": (C.c_int, [_P, _P]),
    "gs_set_tuning": (C.c_int, [_P, _P]),
    "gs_profile_enable": (C.c_int, [_P, C.c_int]),
    "gs_profile_read": (C.c_int, [_P, C.POINTER(GsProfile)]),
    "gs_ingest_pairs_noalloc": (C.c_int, [C.c_uint32, C.c_uint64, C.c_double, _P, C.c_uint64, _P, _P]),
    "gs_engine_create": (C.c_int, [C.POINTER(GsEngineConfig), C.POINTER(_P)]),
    "gs_engine_destroy": (C.c_int, [_P]),
    "gs_engine_tenant_bytes": (C.c_int, [C.c_uint32, C.c_double, _U64P]),
    "gs_engine_add_tenant": (C.c_int, [_P, C.c_uint32, C.c_uint64, C.c_double, _U32P]),
    "gs_engine_remove_tenant": (C.c_int, [_P, C.c_uint32]),
    "gs_engine_clear_tenant": (C.c_int, [_P, C.c_uint32]),
    "gs_engine_memory": (C.c_int, [_P, _U64P, _U64P, _U32P]),
    "gs_engine_set_stream": (C.c_int, [_P, _P]),
    "gs_engine_ingest": (C.c_int, [_P, _P, _P, C.c_uint32, _P, C.c_int, _P]),
    "gs_engine_ingest_slices": (C.c_int, [_P, C.c_uint32, _P, _P, _P, _P]),
    "gs_engine_synchronize": (C.c_int, [_P]),
    "gs_engine_connected_components": (C.c_int, [_P, _P, C.c_uint32, _P, _P, _P]),
    "gs_engine_phase": (C.c_int, [_P, _P, _P, C.c_uint32, _P, _P, C.c_uint32, _P, _P, C.c_int]),
    "gs_engine_graph_stats": (C.c_int, [_P, _U64P, _U64P]),
    "gs_engine_tenant_geometry": (C.c_int, [_P, C.c_uint32, C.POINTER(GsGeometry)]),
    "gs_engine_download_sketches": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, _P]),
    "gs_engine_write_binary": (C.c_int, [_P, C.c_uint32, C.c_char_p]),
    "gs_engine_get_tuning": (C.c_int, [_P, _P]),
    "gs_engine_set_tuning": (C.c_int, [_P, _P]),
    "gs_engine_profile_enable": (C.c_int, [_P, C.c_int]),
    "gs_engine_profile_read": (C.c_int, [_P, C.POINTER(GsProfile)]),
    "gs_last_error": (C.c_char_p, []),
    "gs_gen_er_stream": (C.c_int, [C.c_uint32, C.c_double, C.c_uint64, C.c_double, C.c_double, _P, C.c_uint64, _U64P]),
    "gs_gen_rmat_stream": (C.c_int, [C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                     C.c_uint64, C.c_uint64, _P, C.c_int, _P]),
}

_lib = None


class GpuSketchError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib() -> C.CDLL:
    """Loads libgpusketch_b200.so (RuntimeError when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m gpusketch_b200.build` "
                               "(the package has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != GS_OK:
        raise GpuSketchError(status, where, lib().gs_last_error().decode(errors="replace"))
