// gs_dsu.cuh - lock-free union-find on a device parent array, shared by the Boruvka kernel and the
// eager DSU of the ingest path.
//
// Unions hook the larger root under the smaller with one CAS, so every component's root is its
// minimum vertex id (include/dsu.h:155-167 of the reference unions by random priority instead; the
// partitions are equal).  Every walk is bounded by `limit` steps and sets GS_DEV_ERR_DSU_LIMIT in
// *err instead of looping forever.
#pragma once

#include "gs_common.cuh"

static __device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}

// Root of x.  Path halving: every visited vertex is re-pointed at its grandparent.  Only roots are
// ever CAS'd and a non-root stays a non-root, so these plain stores only ever move a pointer up
// to another ancestor.
static __device__ __forceinline__ uint32_t dsu_find(uint32_t* parent, uint32_t x, uint32_t limit, uint32_t* err) {
  volatile uint32_t* P = parent;
  for (uint32_t it = 0; it < limit; it++) {
    const uint32_t p = P[x];
    if (p == x) return x;
    const uint32_t gp = P[p];
    if (gp != p) P[x] = gp;
    x = gp;
  }
  atomicOr(err, (uint32_t)GS_DEV_ERR_DSU_LIMIT);
  return x;
}

// Root of x without writing anything: the compress phase, where each parent[v] must have exactly
// one writer (thread v).  A path-halving store from another thread could otherwise land after v's
// root and leave v pointing at a non-root.
static __device__ __forceinline__ uint32_t dsu_root(const uint32_t* parent, uint32_t x, uint32_t limit, uint32_t* err) {
  for (uint32_t it = 0; it < limit; it++) {
    const uint32_t p = ld_volatile(parent + x);
    if (p == x) return x;
    x = p;
  }
  atomicOr(err, (uint32_t)GS_DEV_ERR_DSU_LIMIT);
  return x;
}

// union of global vertices a, b; true when it joined two components
static __device__ __forceinline__ bool dsu_union(uint32_t* parent, uint32_t a, uint32_t b, uint32_t limit, uint32_t* err) {
  for (uint32_t it = 0; it < limit; it++) {
    a = dsu_find(parent, a, limit, err);
    b = dsu_find(parent, b, limit, err);
    if (a == b) return false;
    if (a < b) { const uint32_t t = a; a = b; b = t; }
    if (atomicCAS(&parent[a], a, b) == a) return true;
  }
  atomicOr(err, (uint32_t)GS_DEV_ERR_DSU_LIMIT);
  return false;
}

