// gs_boruvka.cu - Boruvka emulation on the device (connected components / spanning forests).
//
// Follows CCSketchAlg::boruvka_emulation (src/cc_sketch_alg.cpp:491-540) round by round:
//   round 0   every vertex samples column `round0_col` of its own sketch (run_round_zero,
//             :250-271; the min-cut forests pass the column their stored sample index reached,
//             src/mc_sketch_alg.cpp:307-328);
//   round r   every current component XORs column r and the deterministic bucket of all its
//             members (Sketch::range_merge, src/sketch.cpp:172-195) and samples column r
//             (perform_boruvka_round, :273-407);
//   sampled edges are unioned into a lock-free DSU; a FAIL sample or a successful union marks
//   the round as modified; the loop stops at the first unmodified round, and a round
//   r >= num_samples is the reference's OutOfSamplesException (src/sketch.cpp:111-113,173-177).
//
// Device mapping:
//   k_sample_*     one warp per supernode: lane j checks bucket j of the column (and j+32) with one
//                  XXH3 each (Bucket_Boruvka::is_good, include/bucket.h:65-67); the sample is the
//                  deterministic bucket when it is zero/good, else the first good bucket by depth,
//                  found with one ballot (Sketch::sample, src/sketch.cpp:110-132).
//   k_accumulate   one warp per vertex of a non-singleton component XORs its column-r slice into
//                  the component accumulator with red.global.xor (the accumulators, 16*(bkt+1) B
//                  per component, stay resident in L2 at the sizes here).
//   k_union        CAS hooking of the larger root under the smaller root; the root of every
//                  component is its minimum vertex id, so labels are deterministic.
//   k_compress     full path compression, so every parent entry is a root after each round.
// Every DSU walk is bounded by V+64 steps and reports GS_DEV_ERR_DSU_LIMIT instead of spinning.
#include "gs_internal.h"

namespace {

constexpr uint32_t kGood = 0, kZero = 1, kFail = 2, kSkip = 3;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ bool is_good(const GsBucket& b, uint64_t csmix) {
  return gs_hash_tail(gs_key_mix(b.alpha) ^ csmix) == b.gamma;
}

// Sketch::sample on one column: all lanes of the warp call it and get the same answer.
__device__ __forceinline__ void sample_warp(const GsBucket* __restrict__ col, const GsBucket* __restrict__ det,
                                            uint32_t bkt, uint64_t csmix, uint32_t* code, uint64_t* idx) {
  const uint32_t lane = lane_id();
  const GsBucket d = *det;
  if (d.alpha == 0 && d.gamma == 0) { *code = kZero; *idx = 0; return; }
  if (is_good(d, csmix)) { *code = kGood; *idx = d.alpha; return; }
  for (uint32_t j0 = 0; j0 < bkt; j0 += 32) {
    const uint32_t j = j0 + lane;
    bool good = false;
    uint64_t a = 0;
    if (j < bkt) {
      const GsBucket b = col[j];
      a = b.alpha;
      good = is_good(b, csmix);
    }
    const uint32_t m = __ballot_sync(0xffffffffu, good);
    if (m) {
      const uint32_t src = __ffs(m) - 1;
      *code = kGood;
      *idx = __shfl_sync(0xffffffffu, a, src);
      return;
    }
  }
  *code = kFail;
  *idx = 0;
}

__device__ __forceinline__ uint32_t ld_parent(const uint32_t* p, uint32_t x) {
  return *reinterpret_cast<const volatile uint32_t*>(p + x);
}

__device__ __forceinline__ uint32_t dsu_find(const uint32_t* parent, uint32_t x, uint32_t limit,
                                             uint32_t* status) {
  for (uint32_t it = 0; it < limit; it++) {
    const uint32_t p = ld_parent(parent, x);
    if (p == x) return x;
    x = p;
  }
  atomicOr(status, (uint32_t)GS_DEV_ERR_DSU_LIMIT);
  return x;
}

__global__ void k_dsu_init(uint32_t* __restrict__ parent, uint32_t V) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) parent[v] = v;
}

__global__ void k_sample_round0(const GsBucket* __restrict__ sk, uint32_t V, uint32_t nb, uint32_t bkt,
                                uint32_t col, uint64_t csmix, uint32_t* __restrict__ res,
                                uint64_t* __restrict__ samp) {
  const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = w0; v < V; v += nw) {
    const GsBucket* base = sk + (size_t)v * nb;
    uint32_t code;
    uint64_t idx;
    sample_warp(base + (size_t)col * bkt, base + (nb - 1), bkt, csmix, &code, &idx);
    if (lane_id() == 0) { res[v] = code; samp[v] = idx; }
  }
}

__global__ void k_sizes(const uint32_t* __restrict__ parent, uint32_t V, uint32_t* __restrict__ size) {
  // lanes with the same root add together: in late rounds most vertices share the giant root
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < V; base += stride) {
    const uint32_t v = base + threadIdx.x;
    const uint32_t r = v < V ? parent[v] : 0xffffffffu;
    const uint32_t peers = __match_any_sync(0xffffffffu, r);
    if (v < V && lane_id() == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&size[r], (uint32_t)__popc(peers));
  }
}

// zero the accumulators of non-singleton roots
__global__ void k_zero_acc(const uint32_t* __restrict__ parent, const uint32_t* __restrict__ size, uint32_t V,
                           uint32_t w, GsBucket* __restrict__ acc) {
  const uint64_t total = (uint64_t)V * w;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)(i / w);
    if (parent[v] == v && size[v] > 1) acc[i] = GsBucket{0, 0};
  }
}

// Each warp walks kAccRun consecutive vertices; lane l holds buckets l, l+32, l+64 of the column-r slice
// (bkt_per_col buckets + the deterministic bucket, at most 65) of the current component in registers
// and flushes them with red.global.xor when the component changes.  Once a giant component has
// formed, runs are long and its accumulator sees one atomic per bucket per run instead of per vertex.
constexpr uint32_t kAccRun = 32;

__device__ __forceinline__ void flush_acc(GsBucket* __restrict__ acc, uint32_t root, uint32_t w, const uint64_t* a,
                                          const uint64_t* g) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint32_t j = lane_id() + 32u * k;
    if (j < w && (a[k] | g[k])) {
      atomicXor(reinterpret_cast<unsigned long long*>(&acc[(size_t)root * w + j].alpha), (unsigned long long)a[k]);
      atomicXor(reinterpret_cast<unsigned long long*>(&acc[(size_t)root * w + j].gamma), (unsigned long long)g[k]);
    }
  }
}

__global__ void k_accumulate(const GsBucket* __restrict__ sk, const uint32_t* __restrict__ parent,
                             const uint32_t* __restrict__ size, uint32_t V, uint32_t nb, uint32_t bkt,
                             uint32_t round, GsBucket* __restrict__ acc) {
  const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t w = bkt + 1;
  for (uint32_t start = w0 * kAccRun; start < V; start += nw * kAccRun) {
    const uint32_t end = min(V, start + kAccRun);
    uint32_t cur = 0xffffffffu;
    uint64_t a[3] = {0, 0, 0}, g[3] = {0, 0, 0};
    for (uint32_t v = start; v < end; v++) {
      const uint32_t root = parent[v];
      if (size[root] <= 1) continue;
      if (root != cur) {
        if (cur != 0xffffffffu) flush_acc(acc, cur, w, a, g);
        cur = root;
#pragma unroll
        for (int k = 0; k < 3; k++) a[k] = g[k] = 0;
      }
      const GsBucket* base = sk + (size_t)v * nb;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const uint32_t j = lane_id() + 32u * k;
        if (j < w) {
          const GsBucket b = j < bkt ? base[(size_t)round * bkt + j] : base[nb - 1];
          a[k] ^= b.alpha;
          g[k] ^= b.gamma;
        }
      }
    }
    if (cur != 0xffffffffu) flush_acc(acc, cur, w, a, g);
  }
}

__global__ void k_sample_roots(const GsBucket* __restrict__ sk, const GsBucket* __restrict__ acc,
                               const uint32_t* __restrict__ parent, const uint32_t* __restrict__ size,
                               uint32_t V, uint32_t nb, uint32_t bkt, uint32_t round, uint64_t csmix,
                               uint32_t* __restrict__ res, uint64_t* __restrict__ samp) {
  const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = w0; v < V; v += nw) {
    uint32_t code = kSkip;
    uint64_t idx = 0;
    if (parent[v] == v) {
      if (size[v] > 1) {
        const GsBucket* a = acc + (size_t)v * (bkt + 1);
        sample_warp(a, a + bkt, bkt, csmix, &code, &idx);
      } else {
        const GsBucket* base = sk + (size_t)v * nb;
        sample_warp(base + (size_t)round * bkt, base + (nb - 1), bkt, csmix, &code, &idx);
      }
    }
    if (lane_id() == 0) { res[v] = code; samp[v] = idx; }
  }
}

// status: [0] error bits, [3] modified flag, [4] forest edge count
__global__ void k_union(const uint32_t* __restrict__ res, const uint64_t* __restrict__ samp, uint32_t V,
                        uint32_t* parent, uint32_t* __restrict__ forest, uint32_t* __restrict__ status) {
  const uint32_t limit = V + 64;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t code = res[v];
    if (code == kFail) { status[3] = 1u; continue; }
    if (code != kGood) continue;
    const uint64_t e = samp[v];
    const uint32_t s = (uint32_t)(e >> 32), d = (uint32_t)e;
    if (s >= V || d >= V || s == d) continue;  // only a checksum collision yields this
    uint32_t a = s, b = d;
    bool merged = false;
    uint32_t it = 0;
    for (; it < limit; it++) {
      a = dsu_find(parent, a, limit, status);
      b = dsu_find(parent, b, limit, status);
      if (a == b) break;
      if (a < b) { const uint32_t t = a; a = b; b = t; }
      if (atomicCAS(&parent[a], a, b) == a) { merged = true; break; }
    }
    if (it == limit) atomicOr(&status[0], (uint32_t)GS_DEV_ERR_DSU_LIMIT);
    if (merged) {
      status[3] = 1u;
      const uint32_t k = atomicAdd(&status[4], 1u);
      if (k + 1 < V + 1) {  // a forest has at most V-1 edges
        forest[2 * k] = min(s, d);
        forest[2 * k + 1] = max(s, d);
      }
    }
  }
}

__global__ void k_compress(uint32_t* parent, uint32_t V, uint32_t* __restrict__ status) {
  const uint32_t limit = V + 64;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t r = dsu_find(parent, v, limit, status);
    parent[v] = r;
  }
}

inline int grid_threads(gs_graph* g, uint64_t items, int threads) {
  uint64_t want = (items + threads - 1) / threads;
  uint64_t cap = (uint64_t)g->num_sms * 16;
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

}  // namespace

gs_status gs_boruvka(gs_graph* g, uint32_t level, uint32_t round0_col, cudaStream_t s) {
  const uint32_t V = g->V, nb = g->geom.num_buckets, bkt = g->geom.bkt_per_col;
  const uint32_t ns = g->geom.num_samples;
  const GsBucket* sk = g->d_sk + (size_t)level * V * nb;
  const uint64_t csmix = gs_seed_mix(g->seed);
  g->labels_valid = false;
  g->last_forest_edges = 0;

  {
    GsProfScope ps(g, GS_PROF_QUERY, s, 1);
    k_dsu_init<<<grid_threads(g, V, 256), 256, 0, s>>>(g->d_parent, V);
  }
  GS_CUDA_TRY(cudaMemsetAsync(g->d_status, 0, 8 * sizeof(uint32_t), s));
  uint32_t round = 0;
  for (;;) {
    GS_CUDA_TRY(cudaMemsetAsync(g->d_status + 3, 0, sizeof(uint32_t), s));
    if (round > 0 && round >= ns) {
      gs_set_error("sketch ran out of samples after " + std::to_string(round) + " Boruvka rounds");
      return GS_ERR_SKETCH_FAIL;
    }
    if (round == 0 && round0_col >= ns) { gs_set_error("sketch out of samples at round 0"); return GS_ERR_SKETCH_FAIL; }
    {
      GsProfScope ps(g, GS_PROF_QUERY, s, round == 0 ? 3 : 6);
      if (round == 0) {
        k_sample_round0<<<grid_threads(g, (uint64_t)V * 32, 256), 256, 0, s>>>(sk, V, nb, bkt, round0_col, csmix,
                                                                               g->d_res, g->d_samp);
      } else {
        GS_CUDA_TRY(cudaMemsetAsync(g->d_size, 0, (size_t)V * sizeof(uint32_t), s));
        k_sizes<<<grid_threads(g, V, 256), 256, 0, s>>>(g->d_parent, V, g->d_size);
        k_zero_acc<<<grid_threads(g, (uint64_t)V * (bkt + 1), 256), 256, 0, s>>>(g->d_parent, g->d_size, V,
                                                                                bkt + 1, g->d_acc);
        k_accumulate<<<grid_threads(g, (uint64_t)(V + kAccRun - 1) / kAccRun * 32, 256), 256, 0, s>>>(
            sk, g->d_parent, g->d_size, V, nb, bkt, round, g->d_acc);
        k_sample_roots<<<grid_threads(g, (uint64_t)V * 32, 256), 256, 0, s>>>(
            sk, g->d_acc, g->d_parent, g->d_size, V, nb, bkt, round, csmix, g->d_res, g->d_samp);
      }
      k_union<<<grid_threads(g, V, 256), 256, 0, s>>>(g->d_res, g->d_samp, V, g->d_parent, g->d_forest,
                                                      g->d_status);
      k_compress<<<grid_threads(g, V, 256), 256, 0, s>>>(g->d_parent, V, g->d_status);
      GS_CUDA_TRY(cudaGetLastError());
    }
    GS_CUDA_TRY(cudaMemcpyAsync(g->h_status, g->d_status, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GS_CUDA_TRY(cudaStreamSynchronize(s));
    if (g->h_status[0] & GS_DEV_ERR_DSU_LIMIT) {
      gs_set_error("DSU walk exceeded its bound");
      return GS_ERR_INTERNAL;
    }
    if (!g->h_status[3]) break;
    round++;
  }
  g->last_rounds = round;
  g->last_forest_edges = g->h_status[4] < V ? g->h_status[4] : (V ? V - 1 : 0);
  g->labels_valid = true;
  g->labels_level = level;
  return GS_OK;
}
