"""Autotuner for the sketch-update launch parameters (records per work item, warps per block,
bucket depths kept in registers).

It times each candidate on the device with the handle's own CUDA-event profile over a sample of the
caller's records, keeps the fastest, and caches the choice per sketch geometry for the process.
Results are bit-identical for every candidate (XOR is order-independent); only speed differs.
"""
from __future__ import annotations

import ctypes as C
import itertools

from ._native import check, lib

_CACHE: dict[tuple, tuple] = {}


class GsTuning(C.Structure):
    _fields_ = [("chunk", C.c_uint32), ("warps_per_block", C.c_uint32), ("reg_depth", C.c_uint32),
                ("reserved", C.c_uint32)]


def _sig():
    return lib()


def _fns(obj):
    """(get, set) entry points for a GraphSketch or a SketchEngine handle."""
    L = _sig()
    if hasattr(obj, "phase"):
        return L.gs_engine_get_tuning, L.gs_engine_set_tuning
    return L.gs_get_tuning, L.gs_set_tuning


def get_tuning(g) -> dict:
    t = GsTuning()
    check(_fns(g)[0](g._h, C.byref(t)), "get_tuning")
    return {"chunk": t.chunk, "warps_per_block": t.warps_per_block, "reg_depth": t.reg_depth}


def set_tuning(g, chunk: int, warps_per_block: int, reg_depth: int) -> None:
    t = GsTuning(chunk, warps_per_block, reg_depth, 0)
    check(_fns(g)[1](g._h, C.byref(t)), "set_tuning")


def autotune(g, sample_pairs, chunks=(256, 512, 1024, 2048), warps=(8, 12, 16), reg_depths=(0, 1),
             repeats: int = 2, table: list | None = None) -> dict:
    """Times every candidate on `sample_pairs` (a CUDA tensor of records) and applies the fastest.
    The sketches are restored afterwards: each candidate ingests the sample twice (XOR cancels)."""
    key = (g.geometry.num_columns, g.geometry.bkt_per_col, int(sample_pairs.shape[0]))
    if key in _CACHE:
        set_tuning(g, *_CACHE[key])
        return dict(zip(("chunk", "warps_per_block", "reg_depth"), _CACHE[key]))
    best, best_ms = None, float("inf")
    for chunk, w, r in itertools.product(chunks, warps, reg_depths):
        set_tuning(g, chunk, w, r)
        g.profile_enable(True)
        for _ in range(repeats):
            g.ingest_pairs(sample_pairs)
            g.ingest_pairs(sample_pairs)
        ms = g.profile_read()["ingest_ms"]
        if table is not None:
            table.append({"chunk": chunk, "warps_per_block": w, "reg_depth": r, "ingest_ms": ms / (2 * repeats)})
        if ms < best_ms:
            best, best_ms = (chunk, w, r), ms
    g.profile_enable(False)
    set_tuning(g, *best)
    _CACHE[key] = best
    return {"chunk": best[0], "warps_per_block": best[1], "reg_depth": best[2], "ingest_ms": best_ms / (2 * repeats)}


def autotune_engine(e, slice_tenants, slice_offsets, pairs, chunks=(128, 256, 512, 1024), warps=(4, 8, 12, 16),
                    reg_depths=(0, 1), repeats: int = 1, table: list | None = None) -> dict:
    """Engine variant: times the multi-tenant sketch update on one batch of device-resident slices
    (ingested twice per candidate, so the tenants' sketches are unchanged) and applies the fastest.
    Tile size = records per work item, vertices per block = warps per block (a warp owns one vertex
    chunk), update-buffer depth = bucket depths kept in registers."""
    best, best_ms = None, float("inf")
    for chunk, w, r in itertools.product(chunks, warps, reg_depths):
        set_tuning(e, chunk, w, r)
        e.profile_enable(True)
        for _ in range(repeats):
            e.ingest(slice_tenants, slice_offsets, pairs)
            e.ingest(slice_tenants, slice_offsets, pairs)
        ms = e.profile_read()["ingest_ms"]
        if table is not None:
            table.append({"chunk": chunk, "warps_per_block": w, "reg_depth": r, "ingest_ms": ms / (2 * repeats)})
        if ms < best_ms:
            best, best_ms = (chunk, w, r), ms
    e.profile_enable(False)
    set_tuning(e, *best)
    return {"chunk": best[0], "warps_per_block": best[1], "reg_depth": best[2], "ingest_ms": best_ms / (2 * repeats)}
