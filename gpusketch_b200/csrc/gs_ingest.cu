// gs_ingest.cu - edge-record ingest: device-side endpoint bucketing + per-vertex sketch update.
//
// Replaces the reference's host gutters + CudaStream double buffering + sketchUpdate kernel
// (include/cuda_stream.h:146-276, src/cuda_kernel.cu:197-257).  One ingest pass over n records:
//
//   1. k_count_*    histogram of records per virtual vertex (level*V + v), warp-aggregated
//                   with __match_any_sync so R-MAT hubs do not serialise on one counter.
//   2. k_scan_*     exclusive scans of the record counts and of the per-vertex work-chunk
//                   counts (ceil(count / chunk)).
//   3. k_scatter_*  each record writes its neighbour id into its vertex's slice of d_nbr.
//   4. k_ingest     one warp per work chunk of one vertex.  Lane c owns sketch column c: for
//                   every record it hashes the edge for its column (XXH3 with the per-column
//                   constant folded, gs_common.cuh) and XORs {edge, checksum} into a
//                   warp-private shared-memory slab holding depths [0, D) of its column.
//                   Only lane c ever touches column c, so the slab needs no atomics and the
//                   padded [depth][33] layout keeps the 16-byte accesses bank-conflict free.
//                   Depths >= D (probability 2^-D per record and column) XOR straight into the
//                   HBM sketch with red.global.xor.  At the end of the chunk the non-zero slab
//                   buckets and the deterministic bucket are merged into the vertex sketch with
//                   coalesced 16-byte read-modify-writes (plain when the vertex is one chunk,
//                   atomic XOR when several warps share it).
//
// XOR is commutative and associative, so the result is bit-identical to the reference's
// sequential Sketch::update over the same records (src/sketch.cpp:85-99), whatever the order.
#include <algorithm>

#include "gs_internal.h"

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanTile = kScanThreads * kScanPer;
constexpr int kSlabDepth = 8;      // depths cached in shared memory per column
constexpr int kSlabPitch = 33;     // 32 lanes + 1 pad: rows land on distinct bank groups

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// lanes of `peers` holding the same key combine their increments; returns the old counter value
// plus this lane's rank among its peers.
__device__ __forceinline__ uint32_t agg_fetch_add(uint32_t* ctr, uint32_t key, bool act) {
  const uint32_t lane = lane_id();
  uint32_t peers = __match_any_sync(0xffffffffu, act ? key : 0xffffffffu);
  uint32_t leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if (act && lane == leader) base = atomicAdd(&ctr[key], (uint32_t)__popc(peers));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}

__device__ __forceinline__ void agg_add(uint32_t* ctr, uint32_t key, bool act) {
  const uint32_t lane = lane_id();
  uint32_t peers = __match_any_sync(0xffffffffu, act ? key : 0xffffffffu);
  if (act && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&ctr[key], (uint32_t)__popc(peers));
}

struct PairTag {
  uint32_t V, num_levels, L;
  int fixed_level;
  uint64_t cs_mix;  // mix(B(seed)): checksum hash constant, also the min-cut tag hash
};

// level range [lo, hi] of a record; returns false when the record is skipped.
__device__ __forceinline__ bool record_levels(const PairTag& t, uint32_t u, uint32_t v, int* lo, int* hi,
                                              uint32_t* status) {
  if (u >= t.V || v >= t.V) {
    atomicOr(status, (uint32_t)GS_DEV_ERR_VERTEX_RANGE);
    return false;
  }
  if (u == v) return false;  // both endpoint updates hit one sketch and cancel
  if (t.fixed_level >= 0) {
    *lo = *hi = t.fixed_level;
  } else if (t.num_levels == 1) {
    *lo = *hi = 0;
  } else {
    // subgraph tag = get_index_depth(e, seed, L-1) (src/mc_gpu_sketch_alg.cpp:160), capped at the
    // deepest sketched level
    uint64_t cs = gs_hash_tail(gs_key_mix(gs_concat(u, v)) ^ t.cs_mix);
    uint64_t hm = cs | (1ull << (t.L - 1));
    int tag = __ffsll((long long)hm) - 1;
    *lo = 0;
    *hi = min(tag, (int)t.num_levels - 1);
  }
  return true;
}

__global__ void k_count_pairs(const uint2* __restrict__ pairs, uint64_t n, PairTag t,
                              uint32_t* __restrict__ cnt, uint32_t* __restrict__ status) {
  const uint64_t warp0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t base = warp0 * 32; base < n; base += nwarps * 32) {
    uint64_t i = base + lane_id();
    int lo = 0, hi = -1;
    uint32_t u = 0, v = 0;
    if (i < n) {
      uint2 p = pairs[i];
      u = p.x; v = p.y;
      if (!record_levels(t, u, v, &lo, &hi, status)) { lo = 0; hi = -1; }
    }
    int wlo = __reduce_min_sync(0xffffffffu, hi >= lo ? lo : 0x7fffffff);
    int whi = __reduce_max_sync(0xffffffffu, hi);
    for (int g = wlo; g <= whi; g++) {
      bool act = g >= lo && g <= hi;
      agg_add(cnt, (uint32_t)g * t.V + u, act);
      agg_add(cnt, (uint32_t)g * t.V + v, act);
    }
  }
}

__global__ void k_scatter_pairs(const uint2* __restrict__ pairs, uint64_t n, PairTag t,
                                uint32_t* __restrict__ cursor, uint32_t* __restrict__ nbr,
                                uint64_t cap, uint32_t* __restrict__ status) {
  const uint64_t warp0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t base = warp0 * 32; base < n; base += nwarps * 32) {
    uint64_t i = base + lane_id();
    int lo = 0, hi = -1;
    uint32_t u = 0, v = 0;
    if (i < n) {
      uint2 p = pairs[i];
      u = p.x; v = p.y;
      // range errors were already reported by the count pass
      if (u >= t.V || v >= t.V || u == v) { hi = -1; }
      else if (!record_levels(t, u, v, &lo, &hi, status)) { lo = 0; hi = -1; }
    }
    int wlo = __reduce_min_sync(0xffffffffu, hi >= lo ? lo : 0x7fffffff);
    int whi = __reduce_max_sync(0xffffffffu, hi);
    for (int g = wlo; g <= whi; g++) {
      bool act = g >= lo && g <= hi;
      uint32_t pu = agg_fetch_add(cursor, (uint32_t)g * t.V + u, act);
      uint32_t pv = agg_fetch_add(cursor, (uint32_t)g * t.V + v, act);
      if (act) {
        if (pu < cap && pv < cap) { nbr[pu] = v; nbr[pv] = u; }
        else atomicOr(status, (uint32_t)GS_DEV_ERR_CAPACITY);
      }
    }
  }
}

// Directed per-vertex batches: batch b adds sizes[b] records to vertex level*V + srcs[b].
__global__ void k_count_batches(const uint32_t* __restrict__ srcs, const uint64_t* __restrict__ sizes,
                                uint32_t nb, uint32_t V, uint32_t level, uint32_t* __restrict__ cnt,
                                uint32_t* __restrict__ status) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    uint32_t s = srcs[b];
    if (s >= V) { atomicOr(status, (uint32_t)GS_DEV_ERR_VERTEX_RANGE); continue; }
    if (sizes[b]) atomicAdd(&cnt[(size_t)level * V + s], (uint32_t)sizes[b]);
  }
}

__global__ void k_scatter_batches(const uint32_t* __restrict__ srcs, const uint64_t* __restrict__ starts,
                                  const uint64_t* __restrict__ sizes, uint32_t nb,
                                  const uint32_t* __restrict__ dsts, uint32_t V, uint32_t level,
                                  uint32_t* __restrict__ cursor, uint32_t* __restrict__ nbr,
                                  uint64_t cap, uint32_t* __restrict__ status) {
  const uint32_t warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t b = warp0; b < nb; b += nwarps) {
    uint32_t s = srcs[b];
    uint64_t sz = sizes[b];
    if (s >= V || sz == 0) continue;
    uint32_t pos = 0;
    if (lane_id() == 0) pos = atomicAdd(&cursor[(size_t)level * V + s], (uint32_t)sz);
    pos = __shfl_sync(0xffffffffu, pos, 0);
    const uint32_t* src = dsts + starts[b];
    for (uint64_t i = lane_id(); i < sz; i += 32) {
      uint32_t d = src[i];
      if (d >= V) { atomicOr(status, (uint32_t)GS_DEV_ERR_VERTEX_RANGE); d = s; }
      if (pos + i < cap) nbr[pos + i] = d;
      else atomicOr(status, (uint32_t)GS_DEV_ERR_CAPACITY);
    }
  }
}

// ---- exclusive scan of (count, ceil(count/chunk)) over nv entries, totals at [nv] ----

__device__ __forceinline__ uint2 add2(uint2 a, uint2 b) { return make_uint2(a.x + b.x, a.y + b.y); }

__device__ uint2 block_exclusive_scan(uint2 x, uint2* total) {
  __shared__ uint2 warp_sums[32];
  __shared__ uint2 block_total;
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  uint2 inc = x;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t a = __shfl_up_sync(0xffffffffu, inc.x, o), b = __shfl_up_sync(0xffffffffu, inc.y, o);
    if (lane >= (uint32_t)o) { inc.x += a; inc.y += b; }
  }
  if (lane == 31) warp_sums[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t nw = blockDim.x >> 5;
    uint2 s = lane < nw ? warp_sums[lane] : make_uint2(0, 0);
    uint2 si = s;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t a = __shfl_up_sync(0xffffffffu, si.x, o), b = __shfl_up_sync(0xffffffffu, si.y, o);
      if (lane >= (uint32_t)o) { si.x += a; si.y += b; }
    }
    if (lane < nw) warp_sums[lane] = make_uint2(si.x - s.x, si.y - s.y);
    if (lane == nw - 1) block_total = si;  // nw <= 32
  }
  __syncthreads();
  uint2 res = add2(warp_sums[w], make_uint2(inc.x - x.x, inc.y - x.y));
  *total = block_total;
  __syncthreads();
  return res;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t* __restrict__ cnt, uint32_t nv,
                                                             uint32_t chunk, uint32_t* __restrict__ off,
                                                             uint32_t* __restrict__ choff,
                                                             uint32_t* __restrict__ tile_sums) {
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanPer;
  uint2 v[kScanPer];
  uint2 s = make_uint2(0, 0);
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    uint64_t i = base + k;
    uint32_t c = i < nv ? cnt[i] : 0u;
    v[k] = make_uint2(c, (c + chunk - 1) / chunk);
    s = add2(s, v[k]);
  }
  uint2 tot;
  uint2 ex = block_exclusive_scan(s, &tot);
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    uint64_t i = base + k;
    if (i < nv) { off[i] = ex.x; choff[i] = ex.y; }
    ex = add2(ex, v[k]);
  }
  if (threadIdx.x == 0) { tile_sums[2 * blockIdx.x] = tot.x; tile_sums[2 * blockIdx.x + 1] = tot.y; }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_top(uint32_t* __restrict__ tile_sums, uint32_t tiles,
                                                           uint32_t* __restrict__ off,
                                                           uint32_t* __restrict__ choff, uint32_t nv,
                                                           uint32_t* __restrict__ status) {
  uint2 carry = make_uint2(0, 0);
  for (uint32_t b0 = 0; b0 < tiles; b0 += kScanThreads) {
    uint32_t i = b0 + threadIdx.x;
    uint2 x = i < tiles ? make_uint2(tile_sums[2 * i], tile_sums[2 * i + 1]) : make_uint2(0, 0);
    uint2 tot;
    uint2 ex = block_exclusive_scan(x, &tot);
    if (i < tiles) { tile_sums[2 * i] = ex.x + carry.x; tile_sums[2 * i + 1] = ex.y + carry.y; }
    carry = add2(carry, tot);
  }
  if (threadIdx.x == 0) {
    off[nv] = carry.x;
    choff[nv] = carry.y;
    status[1] = carry.x;
    status[2] = carry.y;
  }
}

// adds the tile prefixes and resets the counters to the record cursors used by the scatter
__global__ void __launch_bounds__(kScanThreads) k_scan_add(uint32_t* __restrict__ off, uint32_t* __restrict__ choff,
                                                           uint32_t* __restrict__ cursor,
                                                           const uint32_t* __restrict__ tile_sums, uint32_t nv) {
  const uint32_t t = blockIdx.x;
  const uint32_t a = tile_sums[2 * t], b = tile_sums[2 * t + 1];
  const uint64_t base = (uint64_t)t * kScanTile + (uint64_t)threadIdx.x * kScanPer;
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    uint64_t i = base + k;
    if (i < nv) {
      uint32_t o = off[i] + a;
      off[i] = o;
      choff[i] += b;
      cursor[i] = o;
    }
  }
}

// ---- the sketch update ----

struct IngestArgs {
  const uint32_t* off;
  const uint32_t* choff;
  const uint32_t* nbr;
  GsBucket* sk;
  const uint64_t* colmix;   // [C] column constants, [C] = checksum constant
  const uint32_t* status;   // [2] = work chunks
  uint32_t nv, V, C, bkt, nb, chunk;
};

__device__ __forceinline__ void xor_bucket_global(GsBucket* p, uint64_t a, uint64_t g) {
  atomicXor(reinterpret_cast<unsigned long long*>(&p->alpha), (unsigned long long)a);
  atomicXor(reinterpret_cast<unsigned long long*>(&p->gamma), (unsigned long long)g);
}

template <int CG>
__global__ void __launch_bounds__(256) k_ingest(const IngestArgs A) {
  extern __shared__ uint4 smem[];
  constexpr int kSlabWords = CG * kSlabDepth * kSlabPitch;  // uint4 per warp slab
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  uint4* slab = smem + (size_t)wib * (kSlabWords + 32 + 16);
  uint4* rec = slab + kSlabWords;                              // 32 x {mix(k') , checksum}
  uint2* rec_e = reinterpret_cast<uint2*>(rec + 32);           // 32 x edge id

  const uint32_t C = A.C, bkt = A.bkt, nb = A.nb, V = A.V;
  const uint64_t csmix = A.colmix[C];
  uint64_t cmix[CG];
#pragma unroll
  for (int g = 0; g < CG; g++) {
    uint32_t c = lane + 32u * g;
    cmix[g] = c < C ? A.colmix[c] : 0ull;
  }

  const uint32_t total = A.status[2];
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;

  for (uint32_t ch = gw; ch < total; ch += nw) {
    // owner vertex: the largest vv with choff[vv] <= ch (32-way search across the warp)
    uint32_t lo = 0, hi = A.nv;
    while (hi - lo > 1) {
      uint32_t step = (hi - lo + 31) / 32;
      uint32_t probe = lo + (lane + 1) * step;
      bool le = probe < hi && A.choff[probe] <= ch;
      uint32_t k = __popc(__ballot_sync(0xffffffffu, le));
      lo = lo + k * step;
      hi = min(hi, lo + step);
    }
    const uint32_t vv = lo;
    const uint32_t c0 = A.choff[vv];
    const bool exclusive = (A.choff[vv + 1] - c0) == 1;
    const uint32_t rb = A.off[vv] + (ch - c0) * A.chunk;
    const uint32_t re = min(A.off[vv + 1], rb + A.chunk);
    const uint32_t v = vv % V;
    GsBucket* skv = A.sk + (size_t)vv * nb;

    for (int i = lane; i < kSlabWords; i += 32) slab[i] = make_uint4(0, 0, 0, 0);
    uint64_t det_a = 0, det_g = 0;
    __syncwarp();

    for (uint32_t b = rb; b < re; b += 32) {
      const uint32_t r = b + lane;
      const bool valid = r < re;
      const uint32_t u = valid ? A.nbr[r] : v;
      const uint64_t e = gs_concat(v, u);
      const uint64_t E = gs_key_mix(e);
      const uint64_t cs = gs_hash_tail(E ^ csmix);
      if (valid) { det_a ^= e; det_g ^= cs; }
      rec[lane] = make_uint4((uint32_t)E, (uint32_t)(E >> 32), (uint32_t)cs, (uint32_t)(cs >> 32));
      rec_e[lane] = make_uint2((uint32_t)e, (uint32_t)(e >> 32));
      __syncwarp();
      const uint32_t cnt = min(32u, re - b);
      for (uint32_t j = 0; j < cnt; j++) {
        const uint4 q = rec[j];
        const uint2 qe = rec_e[j];
        const uint64_t Ej = ((uint64_t)q.y << 32) | q.x;
#pragma unroll
        for (int g = 0; g < CG; g++) {
          const uint32_t c = lane + 32u * g;
          if (c < C) {
            const uint32_t d = gs_depth_from_mixed(Ej ^ cmix[g], bkt);
            if (d < (uint32_t)kSlabDepth) {
              uint4* p = slab + (g * kSlabDepth + d) * kSlabPitch + lane;
              uint4 t = *p;
              t.x ^= qe.x; t.y ^= qe.y; t.z ^= q.z; t.w ^= q.w;
              *p = t;
            } else if (d < bkt) {
              xor_bucket_global(skv + (size_t)c * bkt + d, ((uint64_t)qe.y << 32) | qe.x,
                                ((uint64_t)q.w << 32) | q.z);
            }
          }
        }
      }
      __syncwarp();
    }

    // merge the slab: item i -> column i / D, depth i % D, so 8 consecutive lanes cover one
    // column's 128 contiguous bytes
#pragma unroll
    for (int g = 0; g < CG; g++) {
      const uint32_t cols = min(32u, C - min(C, 32u * g));
      for (uint32_t i = lane; i < cols * kSlabDepth; i += 32) {
        const uint32_t cl = i / kSlabDepth, d = i % kSlabDepth;
        if (d >= bkt) continue;
        const uint4 t = slab[(g * kSlabDepth + d) * kSlabPitch + cl];
        if ((t.x | t.y | t.z | t.w) == 0u) continue;
        GsBucket* p = skv + (size_t)(cl + 32u * g) * bkt + d;
        const uint64_t a = ((uint64_t)t.y << 32) | t.x, gm = ((uint64_t)t.w << 32) | t.z;
        if (exclusive) {
          uint4* q4 = reinterpret_cast<uint4*>(p);
          uint4 o = *q4;
          o.x ^= t.x; o.y ^= t.y; o.z ^= t.z; o.w ^= t.w;
          *q4 = o;
        } else {
          xor_bucket_global(p, a, gm);
        }
      }
    }
    // deterministic bucket (last bucket of the sketch)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      det_a ^= __shfl_xor_sync(0xffffffffu, det_a, o);
      det_g ^= __shfl_xor_sync(0xffffffffu, det_g, o);
    }
    if (lane == 0 && (det_a | det_g) != 0ull) {
      GsBucket* p = skv + (nb - 1);
      if (exclusive) { p->alpha ^= det_a; p->gamma ^= det_g; }
      else xor_bucket_global(p, det_a, det_g);
    }
    __syncwarp();
  }
}

size_t ingest_smem_bytes(int cg, int warps) {
  return (size_t)warps * (size_t)(cg * kSlabDepth * kSlabPitch + 32 + 16) * sizeof(uint4);
}

template <int CG>
gs_status launch_ingest(gs_graph* g, uint32_t nv, cudaStream_t s) {
  IngestArgs A;
  A.off = g->d_off; A.choff = g->d_choff; A.nbr = g->d_nbr; A.sk = g->d_sk; A.colmix = g->d_colmix;
  A.status = g->d_status; A.nv = nv; A.V = g->V; A.C = g->geom.num_columns;
  A.bkt = g->geom.bkt_per_col; A.nb = g->geom.num_buckets; A.chunk = g->tune.chunk;
  const int warps = (int)g->tune.warps_per_block;
  const size_t smem = ingest_smem_bytes(CG, warps);
  // the opt-in shared-memory limit is a per-device function attribute
  static size_t attr_bytes[64][2] = {};
  if (g->device < 64 && attr_bytes[g->device][CG - 1] < smem) {
    GS_CUDA_TRY(cudaFuncSetAttribute(k_ingest<CG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_bytes[g->device][CG - 1] = smem;
  }
  const int blocks = g->num_sms * (int)g->tune.blocks_per_sm;
  k_ingest<CG><<<blocks, warps * 32, smem, s>>>(A);
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

}  // namespace

gs_status gs_ensure_ingest_scratch(gs_graph* g, uint64_t records) {
  const uint64_t nv = (uint64_t)g->num_levels * g->V;
  if (g->nv_cap < nv) {
    cudaFree(g->d_cnt); cudaFree(g->d_off); cudaFree(g->d_choff); cudaFree(g->d_tile);
    g->d_cnt = g->d_off = g->d_choff = g->d_tile = nullptr;
    const uint64_t tiles = (nv + kScanTile - 1) / kScanTile + 1;
    GS_CUDA_TRY(cudaMalloc(&g->d_cnt, (nv + 1) * sizeof(uint32_t)));
    GS_CUDA_TRY(cudaMalloc(&g->d_off, (nv + 1) * sizeof(uint32_t)));
    GS_CUDA_TRY(cudaMalloc(&g->d_choff, (nv + 1) * sizeof(uint32_t)));
    GS_CUDA_TRY(cudaMalloc(&g->d_tile, 2 * tiles * sizeof(uint32_t)));
    g->nv_cap = nv;
  }
  if (g->nbr_cap < records) {
    cudaFree(g->d_nbr);
    g->d_nbr = nullptr;
    g->nbr_cap = 0;
    GS_CUDA_TRY(cudaMalloc(&g->d_nbr, records * sizeof(uint32_t)));
    g->nbr_cap = records;
  }
  return GS_OK;
}

static gs_status scan_counts(gs_graph* g, uint32_t nv, cudaStream_t s) {
  const uint32_t tiles = (nv + kScanTile - 1) / kScanTile;
  k_scan_tiles<<<tiles, kScanThreads, 0, s>>>(g->d_cnt, nv, g->tune.chunk, g->d_off, g->d_choff, g->d_tile);
  k_scan_top<<<1, kScanThreads, 0, s>>>(g->d_tile, tiles, g->d_off, g->d_choff, nv, g->d_status);
  k_scan_add<<<tiles, kScanThreads, 0, s>>>(g->d_off, g->d_choff, g->d_cnt, g->d_tile, nv);
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

static gs_status ingest_chunks(gs_graph* g, uint32_t nv, cudaStream_t s) {
  if (g->geom.num_columns <= 32) return launch_ingest<1>(g, nv, s);
  if (g->geom.num_columns <= 64) return launch_ingest<2>(g, nv, s);
  gs_set_error("more than 64 sketch columns are not supported");
  return GS_ERR_BAD_ARG;
}

static int grid_for(gs_graph* g, uint64_t work_items, int threads) {
  uint64_t want = (work_items + threads - 1) / threads;
  uint64_t cap = (uint64_t)g->num_sms * 8;
  if (want < 1) want = 1;
  return (int)std::min(want, cap);
}

gs_status gs_ingest_device_pairs(gs_graph* g, const uint32_t* d_pairs, uint64_t n, int fixed_level,
                                 cudaStream_t s) {
  if (n == 0) return GS_OK;
  const uint32_t nv = g->num_levels * g->V;
  PairTag t;
  t.V = g->V; t.num_levels = g->num_levels; t.L = g->num_subgraphs; t.fixed_level = fixed_level;
  t.cs_mix = gs_seed_mix(g->seed);
  const bool tagged = g->num_levels > 1 && fixed_level < 0;
  for (uint64_t done = 0; done < n;) {
    const uint64_t m = std::min<uint64_t>(n - done, g->max_batch_edges);
    const uint2* p = reinterpret_cast<const uint2*>(d_pairs) + done;
    GS_TRY(gs_ensure_ingest_scratch(g, tagged ? g->nbr_cap : 2 * m));
    GS_CUDA_TRY(cudaMemsetAsync(g->d_cnt, 0, (size_t)(nv + 1) * sizeof(uint32_t), s));
    const int grid = grid_for(g, m, 256);
    {
      GsProfScope ps(g, GS_PROF_BUCKET, s, 4);
      k_count_pairs<<<grid, 256, 0, s>>>(p, m, t, g->d_cnt, g->d_status);
      GS_CUDA_TRY(cudaGetLastError());
      GS_TRY(scan_counts(g, nv, s));
    }
    if (tagged) {
      // record count depends on the tags: read it back and grow the scratch if needed
      GS_CUDA_TRY(cudaMemcpyAsync(g->h_status, g->d_status, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      GS_CUDA_TRY(cudaStreamSynchronize(s));
      uint64_t recs = g->h_status[1];
      if (recs > g->nbr_cap) GS_TRY(gs_ensure_ingest_scratch(g, recs + recs / 8));
    }
    {
      GsProfScope ps(g, GS_PROF_BUCKET, s, 1);
      k_scatter_pairs<<<grid, 256, 0, s>>>(p, m, t, g->d_cnt, g->d_nbr, g->nbr_cap, g->d_status);
      GS_CUDA_TRY(cudaGetLastError());
    }
    {
      GsProfScope ps(g, GS_PROF_INGEST, s, 1);
      GS_TRY(ingest_chunks(g, nv, s));
    }
    g->records_total += m;
    done += m;
  }
  return GS_OK;
}

gs_status gs_ingest_device_batches(gs_graph* g, uint32_t level, const uint32_t* d_srcs,
                                   const uint64_t* d_starts, const uint64_t* d_sizes, uint32_t nbat,
                                   const uint32_t* d_dsts, cudaStream_t s) {
  if (nbat == 0) return GS_OK;
  const uint32_t nv = g->num_levels * g->V;
  GS_TRY(gs_ensure_ingest_scratch(g, 1));
  GS_CUDA_TRY(cudaMemsetAsync(g->d_cnt, 0, (size_t)(nv + 1) * sizeof(uint32_t), s));
  {
    GsProfScope ps(g, GS_PROF_BUCKET, s, 4);
    k_count_batches<<<grid_for(g, nbat, 256), 256, 0, s>>>(d_srcs, d_sizes, nbat, g->V, level, g->d_cnt, g->d_status);
    GS_CUDA_TRY(cudaGetLastError());
    GS_TRY(scan_counts(g, nv, s));
  }
  GS_CUDA_TRY(cudaMemcpyAsync(g->h_status, g->d_status, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  const uint64_t recs = g->h_status[1];
  if (recs > g->nbr_cap) GS_TRY(gs_ensure_ingest_scratch(g, recs));
  {
    GsProfScope ps(g, GS_PROF_BUCKET, s, 1);
    k_scatter_batches<<<grid_for(g, (uint64_t)nbat * 32, 256), 256, 0, s>>>(
        d_srcs, d_starts, d_sizes, nbat, d_dsts, g->V, level, g->d_cnt, g->d_nbr, g->nbr_cap, g->d_status);
    GS_CUDA_TRY(cudaGetLastError());
  }
  g->records_total += recs;
  GsProfScope ps(g, GS_PROF_INGEST, s, 1);
  return ingest_chunks(g, nv, s);
}
