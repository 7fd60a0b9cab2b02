"""gpusketch_b200 - B200-native graph-stream sketching (l0 sketches, device Boruvka, k-forest min cut).

The compute path is the in-tree shared library libgpusketch_b200.so (sm_100a kernels behind the C ABI
of include/gpusketch.h); this package binds it with ctypes and mirrors the reference's host classes.
"""
from ._native import GpuSketchError, lib
from .api import (CCAlgConfiguration, CCGPUSketchAlg, CCSketchAlg, ConnectedComponents, Edge, GraphUpdate,
                  MCGPUSketchAlg, MinCut, OutOfSamplesException, QueryCode, SpanningForest, UpdateLockedException,
                  UpdateType)
from .graph import BUCKET_DTYPE, Geometry, GraphSketch, er_stream, exact_min_cut, geometry_for, hash64, rmat_stream

__all__ = [
    "GpuSketchError", "lib", "CCAlgConfiguration", "CCGPUSketchAlg", "CCSketchAlg", "ConnectedComponents", "Edge",
    "GraphUpdate", "MCGPUSketchAlg", "MinCut", "OutOfSamplesException", "QueryCode", "SpanningForest",
    "UpdateLockedException", "UpdateType", "BUCKET_DTYPE", "Geometry", "GraphSketch", "er_stream", "exact_min_cut",
    "geometry_for", "hash64", "rmat_stream",
]
