// gs_eager.cu - eager DSU: connectivity answered without Boruvka while the stream has only grown it.
//
// The reference keeps a DSU and a spanning forest next to the sketches (CCSketchAlg::pre_insert,
// src/cc_sketch_alg.cpp:106-131): every update that joins two components merges them and adds its
// edge to the forest; an update that toggles a forest edge makes the DSU invalid; while it is valid,
// connected_components() answers from the DSU (:542-549, has_cached_query, include/cc_sketch_alg.h:
// 185-191); a Boruvka query makes it valid again with its own forest (:537-538).
//
// Here the DSU is the handle's parent array (after a Boruvka query it already holds the partition)
// and the forest is a device hash set of edge ids.  An ingested batch runs three passes over its raw
// records, concurrently instead of in stream order, and stays conservative:
//   check  a record whose edge is already a forest edge invalidates (it may delete that edge);
//   union  CAS unions; an edge that joins two components enters the set tagged with the batch;
//   dups   an edge that joined components in this batch and occurs more than once in it
//          invalidates (in stream order one of its later toggles would delete a forest edge).
// Every other record either repeats a connection the forest already has (a redundant insert) or
// deletes a non-forest edge, so the partition stays exact.  Once invalid, the passes exit at once.
#include <algorithm>

#include "gs_dsu.cuh"
#include "gs_internal.h"

namespace {

constexpr uint32_t kEagerThreads = 256;

__device__ __forceinline__ uint32_t slot_of(uint64_t key, uint32_t mask) {
  return (uint32_t)gs_hash_tail(key) & mask;
}

// the slot holding `key`, or nullptr; bounded probing
__device__ GsEagerSlot* set_find(GsEagerSlot* set, uint32_t mask, uint64_t key, uint32_t* err) {
  const uint32_t h = slot_of(key, mask);
  for (uint32_t i = 0; i <= mask; i++) {
    GsEagerSlot* s = set + ((h + i) & mask);
    const uint64_t k = *reinterpret_cast<volatile unsigned long long*>(&s->key);
    if (k == key) return s;
    if (k == 0ull) return nullptr;
  }
  atomicOr(err, (uint32_t)GS_DEV_ERR_CAPACITY);
  return nullptr;
}

__device__ void set_insert(GsEagerSlot* set, uint32_t mask, uint64_t key, uint32_t epoch, uint32_t* err) {
  const uint32_t h = slot_of(key, mask);
  for (uint32_t i = 0; i <= mask; i++) {
    GsEagerSlot* s = set + ((h + i) & mask);
    const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(&s->key), 0ull,
                                              (unsigned long long)key);
    if (prev == 0ull) {
      s->epoch = epoch;
      return;
    }
    if (prev == key) return;
  }
  atomicOr(err, (uint32_t)GS_DEV_ERR_CAPACITY);
}

// edge id of a record, or 0 for a record the sketches skip (out of range, self-loop)
__device__ __forceinline__ uint64_t record_key(uint2 p, uint32_t V) {
  if (p.x >= V || p.y >= V || p.x == p.y) return 0ull;
  return gs_concat(p.x, p.y);
}

// st: [0] invalid flag, [1] error bits
__global__ void __launch_bounds__(kEagerThreads) k_eager_check(const uint2* __restrict__ pairs, uint64_t n, uint32_t V,
                                                               GsEagerSlot* set, uint32_t mask, uint32_t* st) {
  if (ld_volatile(&st[0])) return;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t key = record_key(pairs[e], V);
    if (key && set_find(set, mask, key, &st[1])) {
      atomicOr(&st[0], 1u);
      return;
    }
  }
}

__global__ void __launch_bounds__(kEagerThreads) k_eager_union(const uint2* __restrict__ pairs, uint64_t n, uint32_t V,
                                                               uint32_t* parent, GsEagerSlot* set, uint32_t mask,
                                                               uint32_t epoch, uint32_t* st) {
  if (ld_volatile(&st[0])) return;
  const uint32_t limit = V + 64;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 p = pairs[e];
    const uint64_t key = record_key(p, V);
    if (key && dsu_union(parent, p.x, p.y, limit, &st[1])) set_insert(set, mask, key, epoch, &st[1]);
  }
}

__global__ void __launch_bounds__(kEagerThreads) k_eager_dups(const uint2* __restrict__ pairs, uint64_t n, uint32_t V,
                                                              GsEagerSlot* set, uint32_t mask, uint32_t epoch,
                                                              uint32_t* st) {
  if (ld_volatile(&st[0])) return;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t key = record_key(pairs[e], V);
    if (!key) continue;
    GsEagerSlot* s = set_find(set, mask, key, &st[1]);
    if (s && s->epoch == epoch && atomicAdd(&s->count, 1u) >= 1u) atomicOr(&st[0], 1u);
  }
}

__global__ void k_eager_reset_parent(uint32_t* parent, uint32_t V) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) parent[v] = v;
}

// parent[v] = root(v): each entry has one writer, and every walk only reads
__global__ void k_eager_compress(uint32_t* parent, uint32_t V, uint32_t* st) {
  const uint32_t limit = V + 64;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    parent[v] = dsu_root(parent, v, limit, &st[1]);
}

// the forest set from a Boruvka forest (edge endpoints as (min, max) pairs)
__global__ void k_eager_load_forest(const uint32_t* __restrict__ forest, uint32_t m, GsEagerSlot* set, uint32_t mask,
                                    uint32_t* st) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    set_insert(set, mask, gs_concat(forest[2 * i], forest[2 * i + 1]), 0u, &st[1]);
}

// the set's edges into forest[] (order unspecified); st[2] counts them
__global__ void k_eager_dump_forest(const GsEagerSlot* __restrict__ set, uint32_t slots, uint32_t* forest,
                                    uint32_t cap, uint32_t* st) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < slots; i += gridDim.x * blockDim.x) {
    const uint64_t k = set[i].key;
    if (!k) continue;
    const uint32_t at = atomicAdd(&st[2], 1u);
    if (at < cap) {
      forest[2 * at] = (uint32_t)(k >> 32);
      forest[2 * at + 1] = (uint32_t)k;
    }
  }
}

int grid_for_items(const gs_graph* g, uint64_t items) {
  const uint64_t want = (items + kEagerThreads - 1) / kEagerThreads;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)g->num_sms * 8));
}

}  // namespace

gs_status gs_eager_enable(gs_graph* g, bool on, cudaStream_t s) {
  if (!on) {
    g->eager_on = false;
    return GS_OK;
  }
  if (g->num_levels != 1) {
    gs_set_error("the eager DSU serves connected-components graphs (num_levels == 1)");
    return GS_ERR_BAD_ARG;
  }
  if (!g->d_eager_set) {
    uint32_t slots = 1024;
    while (slots < 4ull * g->V) slots <<= 1;  // forest edges < V: the set stays under a quarter full
    GS_CUDA_TRY(cudaMalloc(&g->d_eager_set, (size_t)slots * sizeof(GsEagerSlot)));
    GS_CUDA_TRY(cudaMalloc(&g->d_eager_status, 4 * sizeof(uint32_t)));
    GS_CUDA_TRY(cudaMallocHost(&g->h_eager, 4 * sizeof(uint32_t)));
    g->eager_mask = slots - 1;
  }
  g->eager_on = true;
  // a handle that has ingested nothing is the empty graph, whose DSU is all singletons; otherwise the
  // next query rebuilds the DSU with a Boruvka run
  if (g->records_total == 0) return gs_eager_reset_empty(g, s);
  GS_CUDA_TRY(cudaMemsetAsync(g->d_eager_status, 0, 4 * sizeof(uint32_t), s));
  return gs_eager_invalidate(g, s);
}

gs_status gs_eager_reset_empty(gs_graph* g, cudaStream_t s) {
  if (!g->eager_on) return GS_OK;
  GS_CUDA_TRY(cudaMemsetAsync(g->d_eager_set, 0, ((size_t)g->eager_mask + 1) * sizeof(GsEagerSlot), s));
  GS_CUDA_TRY(cudaMemsetAsync(g->d_eager_status, 0, 4 * sizeof(uint32_t), s));
  k_eager_reset_parent<<<grid_for_items(g, g->V), kEagerThreads, 0, s>>>(g->d_parent, g->V);
  GS_CUDA_TRY(cudaGetLastError());
  g->eager_epoch = 0;
  g->labels_valid = false;
  return GS_OK;
}

gs_status gs_eager_invalidate(gs_graph* g, cudaStream_t s) {
  if (!g->eager_on) return GS_OK;
  // any non-zero value in word 0 means invalid
  GS_CUDA_TRY(cudaMemsetAsync(g->d_eager_status, 0xff, sizeof(uint32_t), s));
  return GS_OK;
}

gs_status gs_eager_ingest(gs_graph* g, const uint32_t* d_pairs, uint64_t n, cudaStream_t s) {
  if (!g->eager_on || n == 0) return GS_OK;
  const uint2* p = reinterpret_cast<const uint2*>(d_pairs);
  const uint32_t epoch = ++g->eager_epoch;
  const int grid = grid_for_items(g, n);
  GsProfScope ps(g, GS_PROF_BUCKET, s, 3);
  k_eager_check<<<grid, kEagerThreads, 0, s>>>(p, n, g->V, g->d_eager_set, g->eager_mask, g->d_eager_status);
  k_eager_union<<<grid, kEagerThreads, 0, s>>>(p, n, g->V, g->d_parent, g->d_eager_set, g->eager_mask, epoch,
                                               g->d_eager_status);
  k_eager_dups<<<grid, kEagerThreads, 0, s>>>(p, n, g->V, g->d_eager_set, g->eager_mask, epoch, g->d_eager_status);
  GS_CUDA_TRY(cudaGetLastError());
  g->labels_valid = false;
  return GS_OK;
}

gs_status gs_eager_state(gs_graph* g, cudaStream_t s, bool* valid) {
  *valid = false;
  if (!g->eager_on) return GS_OK;
  GS_CUDA_TRY(cudaMemcpyAsync(g->h_eager, g->d_eager_status, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  if (g->h_eager[1] & GS_DEV_ERR_DSU_LIMIT) {
    gs_set_error("eager DSU walk exceeded its bound");
    return GS_ERR_INTERNAL;
  }
  if (g->h_eager[1] & GS_DEV_ERR_CAPACITY) {
    gs_set_error("eager DSU forest set overflowed");
    return GS_ERR_INTERNAL;
  }
  *valid = g->h_eager[0] == 0;
  return GS_OK;
}

gs_status gs_eager_answer(gs_graph* g, cudaStream_t s) {
  k_eager_compress<<<grid_for_items(g, g->V), kEagerThreads, 0, s>>>(g->d_parent, g->V, g->d_eager_status);
  GS_CUDA_TRY(cudaGetLastError());
  g->last_rounds = 0;
  g->last_answer_eager = true;
  g->labels_valid = true;
  g->labels_level = 0;
  g->eager_answers++;
  return GS_OK;
}

gs_status gs_eager_rebuild(gs_graph* g, cudaStream_t s) {
  if (!g->eager_on) return GS_OK;
  // d_parent holds the Boruvka partition; its forest becomes the eager forest
  GS_CUDA_TRY(cudaMemsetAsync(g->d_eager_set, 0, ((size_t)g->eager_mask + 1) * sizeof(GsEagerSlot), s));
  GS_CUDA_TRY(cudaMemsetAsync(g->d_eager_status, 0, 4 * sizeof(uint32_t), s));
  if (g->last_forest_edges) {
    k_eager_load_forest<<<grid_for_items(g, g->last_forest_edges), kEagerThreads, 0, s>>>(
        g->d_forest, g->last_forest_edges, g->d_eager_set, g->eager_mask, g->d_eager_status);
    GS_CUDA_TRY(cudaGetLastError());
  }
  g->eager_epoch = 0;
  return GS_OK;
}

gs_status gs_eager_forest(gs_graph* g, cudaStream_t s) {
  GS_CUDA_TRY(cudaMemsetAsync(g->d_eager_status + 2, 0, sizeof(uint32_t), s));
  k_eager_dump_forest<<<grid_for_items(g, (uint64_t)g->eager_mask + 1), kEagerThreads, 0, s>>>(
      g->d_eager_set, g->eager_mask + 1, g->d_forest, g->V, g->d_eager_status);
  GS_CUDA_TRY(cudaGetLastError());
  GS_CUDA_TRY(cudaMemcpyAsync(g->h_eager + 2, g->d_eager_status + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  const uint32_t m = g->h_eager[2];
  g->last_forest_edges = m < g->V ? m : g->V - 1;
  return GS_OK;
}
