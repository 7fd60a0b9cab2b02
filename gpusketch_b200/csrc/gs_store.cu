// gs_store.cu - exact tier for the deep subgraph levels of a min-cut graph.
//
// A min-cut graph tags every edge with the subgraph depth get_index_depth(e, seed, L-1)
// (src/mc_gpu_sketch_alg.cpp:139-178 of the reference) and keeps sketches for the first store_first
// depths.  Edges whose tag reaches store_first also belong to deeper subgraphs that no sketch level
// holds; the reference keeps them exactly in its EdgeStore (src/edge_store.cpp:60-300: a sorted
// per-vertex adjacency in which a second toggle of an edge deletes it) and answers the first
// unsketched level of the min-cut driver from it (tools/min_cut.cu:208-252).
//
// Here that tier is a device hash set keyed by edge id.  Each slot keeps the edge's tag and the
// parity of its toggles, so a record flips its edge's presence exactly as the reference's merge does;
// st[0] counts the present edges.  One pass over every tagged ingest batch feeds it; the driver reads
// the live edges of a level back.
//
// Adaptive tier (gs_graph_set_edge_store): the graph starts with store_first = initial sketched levels
// and a budget of present edges (the reference's EdgeStore max_edges = sketch_bytes / 8 directed
// entries, i.e. sketch_bytes / 16 edges, src/edge_store.cpp:8-16).  After each ingest pass, when the
// store holds at least the budget and a sketch level is free, its lowest level becomes a sketch level,
// as the reference's check_if_too_big / vertex_contract do (src/edge_store.cpp:212-300): every present
// stored edge is XORed into sketch level store_first (each has tag >= store_first, so it belongs to
// that level), store_first grows by one, and the store is rebuilt from the edges whose tag passes the
// new store_first.  Without gs_graph_set_edge_store every configured level is a sketch from the start.
#include <algorithm>

#include "gs_internal.h"

namespace {

constexpr uint32_t kStoreThreads = 256;

__device__ __forceinline__ uint32_t store_slot(uint64_t key, uint32_t mask) {
  return (uint32_t)gs_hash_tail(key) & mask;
}

// flips the presence of edge `key` (tag `tag`); bounded probing, overflow reported in st[1]
__global__ void __launch_bounds__(kStoreThreads) k_store_toggle(const uint2* __restrict__ pairs, uint64_t n, uint32_t V,
                                                                uint32_t L, uint64_t cs_mix, uint32_t first,
                                                                GsStoreSlot* set, uint32_t mask, uint32_t* st) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 p = pairs[e];
    if (p.x >= V || p.y >= V || p.x == p.y) continue;
    const uint64_t key = gs_concat(p.x, p.y);
    // the subgraph tag, as the ingest path computes it (record_levels in gs_ingest.cu)
    const uint64_t cs = gs_hash_tail(gs_key_mix(key) ^ cs_mix);
    const uint32_t tag = (uint32_t)(__ffsll((long long)(cs | (1ull << (L - 1)))) - 1);
    if (tag < first) continue;
    const uint32_t h = store_slot(key, mask);
    bool placed = false;
    for (uint32_t i = 0; i <= mask; i++) {
      GsStoreSlot* s = set + ((h + i) & mask);
      const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(&s->key), 0ull,
                                                (unsigned long long)key);
      if (prev == 0ull || prev == key) {
        if (prev == 0ull) {
          s->tag = tag;
          atomicAdd(&st[2], 1u);
        }
        // st[0]: present edges (an odd parity means present)
        if (atomicXor(&s->parity, 1u) & 1u) atomicSub(&st[0], 1u);
        else atomicAdd(&st[0], 1u);
        placed = true;
        break;
      }
    }
    if (!placed) atomicOr(&st[1], (uint32_t)GS_DEV_ERR_CAPACITY);
  }
}

// live edges (odd parity) with tag >= min_tag, as (min, max) pairs; st[3] counts them
__global__ void k_store_collect(const GsStoreSlot* __restrict__ set, uint32_t slots, uint32_t min_tag,
                                uint32_t* out, uint64_t cap, uint32_t* st) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < slots; i += gridDim.x * blockDim.x) {
    const GsStoreSlot s = set[i];
    if (!s.key || !(s.parity & 1u) || s.tag < min_tag) continue;
    const uint32_t at = atomicAdd(&st[3], 1u);
    if (at < cap) {
      out[2 * (uint64_t)at] = (uint32_t)(s.key >> 32);
      out[2 * (uint64_t)at + 1] = (uint32_t)s.key;
    }
  }
}

int store_grid(const gs_graph* g, uint64_t items) {
  const uint64_t want = (items + kStoreThreads - 1) / kStoreThreads;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)g->num_sms * 8));
}

}  // namespace

bool gs_store_active(const gs_graph* g) { return g->num_subgraphs > g->store_first; }

gs_status gs_store_ingest(gs_graph* g, const uint32_t* d_pairs, uint64_t n, cudaStream_t s) {
  if (!gs_store_active(g) || n == 0) return GS_OK;
  if (!g->d_store) {
    // a fixed tier holds as many edges as one sketch level has bytes at 16 bytes per edge (the
    // reference's EdgeStore bound before it contracts), at most half full; an adaptive one four times
    // its budget, so the slots left by deleted edges and one pass's growth past the budget fit until
    // the pass ends and the tier contracts or compacts
    const uint64_t level_bytes = (uint64_t)g->V * g->geom.num_buckets * sizeof(GsBucket);
    const uint64_t want = g->store_adaptive ? 4 * g->store_budget : 2 * (level_bytes / 16);
    uint64_t slots = 1u << 16;
    while (slots < want && slots < (1ull << 31)) slots <<= 1;
    GS_CUDA_TRY(cudaMalloc(&g->d_store, slots * sizeof(GsStoreSlot)));
    GS_CUDA_TRY(cudaMemsetAsync(g->d_store, 0, slots * sizeof(GsStoreSlot), s));
    if (!g->d_store_status) {
      GS_CUDA_TRY(cudaMalloc(&g->d_store_status, 4 * sizeof(uint32_t)));
      GS_CUDA_TRY(cudaMallocHost(&g->h_store, 4 * sizeof(uint32_t)));
    }
    GS_CUDA_TRY(cudaMemsetAsync(g->d_store_status, 0, 4 * sizeof(uint32_t), s));
    g->store_mask = (uint32_t)(slots - 1);
  }
  GsProfScope ps(g, GS_PROF_BUCKET, s, 1);
  k_store_toggle<<<store_grid(g, n), kStoreThreads, 0, s>>>(reinterpret_cast<const uint2*>(d_pairs), n, g->V,
                                                             g->num_subgraphs, gs_seed_mix(g->seed), g->store_first,
                                                             g->d_store, g->store_mask, g->d_store_status);
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

gs_status gs_store_maintain(gs_graph* g, cudaStream_t s) {
  if (!g->store_adaptive || !g->d_store) return GS_OK;
  const uint32_t slots = g->store_mask + 1;
  for (;;) {
    GS_CUDA_TRY(cudaMemcpyAsync(g->h_store, g->d_store_status, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GS_CUDA_TRY(cudaStreamSynchronize(s));
    if (g->h_store[1] & GS_DEV_ERR_CAPACITY) {
      gs_set_error("edge store overflowed within one ingest pass: give the graph a larger store budget or smaller passes");
      return GS_ERR_OOM;
    }
    const uint64_t live = g->h_store[0], used = g->h_store[2];
    const bool contract = live >= g->store_budget && g->store_first < g->num_levels;
    const bool compact = !contract && used > slots / 2;
    if (!contract && !compact) return GS_OK;
    // every present edge of the store, into a list
    if (g->store_list_cap < std::max<uint64_t>(live, 1)) {
      cudaFree(g->d_store_list);
      g->d_store_list = nullptr;
      g->store_list_cap = 0;
      GS_CUDA_TRY(cudaMalloc(&g->d_store_list, std::max<uint64_t>(live, 1) * sizeof(uint2)));
      g->store_list_cap = std::max<uint64_t>(live, 1);
    }
    GS_CUDA_TRY(cudaMemsetAsync(g->d_store_status + 3, 0, sizeof(uint32_t), s));
    k_store_collect<<<store_grid(g, slots), kStoreThreads, 0, s>>>(g->d_store, slots, g->store_first,
                                                                   reinterpret_cast<uint32_t*>(g->d_store_list),
                                                                   live, g->d_store_status);
    GS_CUDA_TRY(cudaGetLastError());
    if (contract) {
      // the lowest stored level becomes a sketch level: all stored edges belong to it
      GS_TRY(gs_ingest_device_pairs(g, reinterpret_cast<const uint32_t*>(g->d_store_list), live, (int)g->store_first, s));
      g->store_first++;
      g->store_contractions++;
    }
    // rebuild the store from the edges whose tag passes the sketched levels (parity 1 each)
    GS_CUDA_TRY(cudaMemsetAsync(g->d_store, 0, (size_t)slots * sizeof(GsStoreSlot), s));
    GS_CUDA_TRY(cudaMemsetAsync(g->d_store_status, 0, 4 * sizeof(uint32_t), s));
    if (live) {
      k_store_toggle<<<store_grid(g, live), kStoreThreads, 0, s>>>(g->d_store_list, live, g->V, g->num_subgraphs,
                                                                    gs_seed_mix(g->seed), g->store_first, g->d_store,
                                                                    g->store_mask, g->d_store_status);
      GS_CUDA_TRY(cudaGetLastError());
    }
    if (!contract) {
      // a compaction that still leaves the table over half full cannot help the next pass
      GS_CUDA_TRY(cudaMemcpyAsync(g->h_store, g->d_store_status, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      GS_CUDA_TRY(cudaStreamSynchronize(s));
      return GS_OK;
    }
  }
}

gs_status gs_store_clear(gs_graph* g, cudaStream_t s) {
  if (!g->d_store) return GS_OK;
  GS_CUDA_TRY(cudaMemsetAsync(g->d_store, 0, ((size_t)g->store_mask + 1) * sizeof(GsStoreSlot), s));
  GS_CUDA_TRY(cudaMemsetAsync(g->d_store_status, 0, 4 * sizeof(uint32_t), s));
  return GS_OK;
}

gs_status gs_store_edges(gs_graph* g, uint32_t min_tag, std::vector<uint32_t>* out, cudaStream_t s) {
  out->clear();
  if (!g->d_store) return GS_OK;
  const uint32_t slots = g->store_mask + 1;
  for (int pass = 0; pass < 2; pass++) {
    // first pass counts, second copies into a buffer of that size
    const uint64_t cap = pass == 0 ? 0 : out->size() / 2;
    uint32_t* d_out = nullptr;
    if (cap) GS_CUDA_TRY(cudaMalloc(&d_out, cap * 2 * sizeof(uint32_t)));
    GS_CUDA_TRY(cudaMemsetAsync(g->d_store_status + 3, 0, sizeof(uint32_t), s));
    k_store_collect<<<store_grid(g, slots), kStoreThreads, 0, s>>>(g->d_store, slots, min_tag, d_out, cap,
                                                                   g->d_store_status);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->h_store, g->d_store_status, 4 * sizeof(uint32_t),
                                              cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && cap) e = cudaMemcpy(out->data(), d_out, cap * 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    cudaFree(d_out);
    if (e != cudaSuccess) {
      gs_set_error(std::string("edge store read-back: ") + cudaGetErrorString(e));
      return GS_ERR_CUDA;
    }
    if (g->h_store[1] & GS_DEV_ERR_CAPACITY) {
      gs_set_error("edge store overflowed: give the graph more sketch levels");
      return GS_ERR_OOM;
    }
    if (pass == 0) out->resize((size_t)g->h_store[3] * 2);
    if (out->empty()) break;
  }
  return GS_OK;
}
