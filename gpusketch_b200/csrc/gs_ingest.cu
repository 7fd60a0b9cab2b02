// gs_ingest.cu - edge-record ingest: device-side endpoint bucketing + per-vertex sketch update.
//
// Replaces the reference's host gutters + CudaStream double buffering + sketchUpdate kernel
// (include/cuda_stream.h:146-276, src/cuda_kernel.cu:197-257).  One ingest pass over n records:
//
//   1. k_part_count / k_part_scan    per block, a shared-memory histogram of the records' keys
//                                    (level*V + v) >> lb; one global atomic per non-empty bucket
//   2. k_part_scatter(_staged)       records placed by bucket: sorted per block in shared memory,
//                                    then written as coalesced runs
//   3. k_vert_count, k_scan_*        per-vertex record counts and work chunks ceil(count / chunk)
//   4. k_vert_scatter(_sorted)       neighbours placed by vertex inside each chunk of a bucket
//   5. k_ingest_packed / k_ingest    one warp per work chunk of one vertex.  A lane hashes the edge
//                                    for one column (XXH3 with the column constant folded,
//                                    gs_common.cuh) and XORs {mix(edge), checksum} into the
//                                    shared-memory row of that column and depth (depths < 10);
//                                    deeper buckets (probability 2^-10) go straight to HBM with
//                                    red.global.xor.  k_ingest_packed (at most 24 columns with the
//                                    packed layout, up to 32 without) covers the columns of four
//                                    records with 32 lanes in three steps; k_ingest (wider sketches,
//                                    register depths) keeps lane = column.  At the end of the chunk
//                                    the non-zero rows and the deterministic bucket are merged into
//                                    the vertex sketch (plain read-modify-write when the vertex is
//                                    one chunk, atomic XOR when several warps share it).
//
// XOR is commutative and associative, so the result is bit-identical to the reference's
// sequential Sketch::update over the same records (src/sketch.cpp:85-99), whatever the order.
#include <algorithm>

#include "gs_internal.h"

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanTile = kScanThreads * kScanPer;
constexpr int kSlabDepth = 10;     // depths [R, 10) in a lane-private shared-memory row
constexpr int kSlabPitch = 32;     // lane L's rows stay in bank group L % 8: a quarter-warp's row
                                   // accesses never conflict, whatever depths its lanes hit

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Shared-memory slot counter: the old value of hist[key] (the record's place among its key's
// records), nothing for invalid lanes.
__device__ __forceinline__ uint32_t slot_inc(uint32_t* hist, uint32_t key, bool valid) {
  return valid ? atomicAdd(&hist[key], 1u) : 0u;
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

// ---- two-level counting sort of the records by virtual vertex ----
//
// Pass 1 partitions the records by the high bits of their key (key >> LB, at most kMaxBuckets
// buckets), pass 2 counts and places them by vertex inside each bucket.  Every histogram lives in
// shared memory; global atomics happen once per (block, non-empty bucket) and once per (block,
// non-empty vertex), so hub vertices of skewed streams cost no more than any other vertex.

constexpr int kPartThreads = 512;
constexpr int kPartEdges = 4096;      // edges per block in pass 1
constexpr int kVertChunk = 8192;      // partitioned records per block iteration in pass 2
constexpr int kMaxBuckets = 4096;
constexpr int kVertUnroll = 8;        // records a pass-2 thread loads before its shared-memory atomics
constexpr uint64_t kMaxBlockHistWords = 1ull << 24;  // per-block bucket counts kept between pass-1 kernels (64 MB)
constexpr uint64_t kMaxChunkHistWords = 1ull << 25;  // per-chunk vertex counts kept between pass-2 kernels (128 MB)

// blockhist (may be null): the block's own histogram is also stored at [blockIdx.x * H], so that the
// staged placement of the same block need not count its edges again
__global__ void __launch_bounds__(kPartThreads) k_part_count(const uint2* __restrict__ pairs, uint64_t n, PairTag t,
                                                             uint32_t lb, uint32_t H, uint32_t* __restrict__ tot,
                                                             uint32_t* __restrict__ status,
                                                             uint32_t* __restrict__ blockhist) {
  extern __shared__ uint32_t hist[];
  for (uint32_t i = threadIdx.x; i < H; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const uint64_t e0 = (uint64_t)blockIdx.x * kPartEdges;
  const uint64_t e1 = min(n, e0 + kPartEdges);
  for (uint64_t b = e0; b < e1; b += (uint64_t)blockDim.x * kVertUnroll) {
    uint2 ps[kVertUnroll];
#pragma unroll
    for (int j = 0; j < kVertUnroll; j++) {
      const uint64_t e = b + threadIdx.x + (uint64_t)j * blockDim.x;
      ps[j] = e < e1 ? pairs[e] : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int j = 0; j < kVertUnroll; j++) {
      const uint64_t e = b + threadIdx.x + (uint64_t)j * blockDim.x;
      if (e >= e1) continue;
      const uint2 p = ps[j];
      int lo = 0, hi = -1;
      if (!record_levels(t, p.x, p.y, &lo, &hi, status)) continue;
      for (int g = lo; g <= hi; g++) {
        atomicAdd(&hist[((uint32_t)g * t.V + p.x) >> lb], 1u);
        atomicAdd(&hist[((uint32_t)g * t.V + p.y) >> lb], 1u);
      }
    }
  }
  __syncthreads();
  for (uint32_t d = threadIdx.x; d < H; d += blockDim.x) {
    if (hist[d]) atomicAdd(&tot[d], hist[d]);
    if (blockhist) blockhist[(size_t)blockIdx.x * H + d] = hist[d];
  }
}

// bkt layout: tot[H] | off[H+1] | cur[H] | choff[H+1]; status[1] = records, status[5] = pass-2 chunks
__global__ void __launch_bounds__(kScanThreads) k_part_scan(uint32_t* __restrict__ bkt, uint32_t H,
                                                            uint32_t* __restrict__ status) {
  uint32_t* tot = bkt;
  uint32_t* off = bkt + H;
  uint32_t* cur = off + H + 1;
  uint32_t* choff = cur + H;
  uint2 carry = make_uint2(0, 0);
  for (uint32_t b0 = 0; b0 < H; b0 += kScanThreads) {
    const uint32_t d = b0 + threadIdx.x;
    const uint32_t c = d < H ? tot[d] : 0u;
    const uint2 x = make_uint2(c, (c + kVertChunk - 1) / kVertChunk);
    uint2 total;
    const uint2 ex = block_exclusive_scan(x, &total);
    if (d < H) {
      off[d] = ex.x + carry.x;
      cur[d] = ex.x + carry.x;
      choff[d] = ex.y + carry.y;
    }
    carry = add2(carry, total);
  }
  if (threadIdx.x == 0) {
    off[H] = carry.x;
    choff[H] = carry.y;
    status[1] = carry.x;
    status[5] = carry.y;
  }
}

__global__ void __launch_bounds__(kPartThreads) k_part_scatter(const uint2* __restrict__ pairs, uint64_t n, PairTag t,
                                                               uint32_t lb, uint32_t H, uint32_t* __restrict__ bkt,
                                                               uint2* __restrict__ part, uint64_t cap,
                                                               uint32_t* __restrict__ status) {
  extern __shared__ uint32_t sh[];
  uint32_t* hist = sh;
  uint32_t* base = sh + H;
  uint32_t* cur = bkt + 2 * H + 1;
  for (uint32_t i = threadIdx.x; i < H; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const uint64_t e0 = (uint64_t)blockIdx.x * kPartEdges;
  const uint64_t e1 = min(n, e0 + kPartEdges);
  PairTag quiet = t;
  for (uint64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const uint2 p = pairs[e];
    if (p.x >= t.V || p.y >= t.V) continue;  // reported by k_part_count
    int lo = 0, hi = -1;
    if (!record_levels(quiet, p.x, p.y, &lo, &hi, status)) continue;
    for (int g = lo; g <= hi; g++) {
      atomicAdd(&hist[((uint32_t)g * t.V + p.x) >> lb], 1u);
      atomicAdd(&hist[((uint32_t)g * t.V + p.y) >> lb], 1u);
    }
  }
  __syncthreads();
  for (uint32_t d = threadIdx.x; d < H; d += blockDim.x) {
    const uint32_t c = hist[d];
    base[d] = c ? atomicAdd(&cur[d], c) : 0u;
    hist[d] = 0;
  }
  __syncthreads();
  for (uint64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const uint2 p = pairs[e];
    if (p.x >= t.V || p.y >= t.V) continue;
    int lo = 0, hi = -1;
    if (!record_levels(quiet, p.x, p.y, &lo, &hi, status)) continue;
    for (int g = lo; g <= hi; g++) {
      const uint32_t ku = (uint32_t)g * t.V + p.x, kv = (uint32_t)g * t.V + p.y;
      const uint32_t pu = base[ku >> lb] + atomicAdd(&hist[ku >> lb], 1u);
      const uint32_t pv = base[kv >> lb] + atomicAdd(&hist[kv >> lb], 1u);
      if (pu < cap && pv < cap) {
        part[pu] = make_uint2(ku, p.y);
        part[pv] = make_uint2(kv, p.x);
      } else {
        atomicOr(status, (uint32_t)GS_DEV_ERR_CAPACITY);
      }
    }
  }
}

// Pass 1 placement when every edge makes exactly two records (one level).  Pass A counts the block's
// records per bucket in shared memory; after the block scan and the global range
// reservation, pass B reads the edges again (from L2: the block read them a moment ago) and takes each
// record's place in the block's bucket-sorted shared stage from a cursor; the stage is then written
// out with consecutive threads on consecutive addresses of each bucket's run.  Nothing is held in
// registers across the scan.
size_t part_scatter_staged_smem(uint32_t H) {
  return (size_t)((4 * H + 1 + 1) & ~1u) * sizeof(uint32_t) + (size_t)2 * kPartEdges * sizeof(uint2);
}

//
// COMPACT: the records leave as one word, (key & (2^lb - 1)) << (32 - lb) | neighbour, which holds
// both whenever every neighbour id is below 2^(32 - lb) (V = 2^17: 9 + 17 bits); pass 2 then reads
// 4 bytes per record instead of 8.
template <bool COMPACT>
__global__ void __launch_bounds__(kPartThreads, 3) k_part_scatter_staged(const uint2* __restrict__ pairs, uint64_t n,
                                                                      PairTag t, uint32_t lb, uint32_t H,
                                                                      uint32_t* __restrict__ bkt,
                                                                      uint2* __restrict__ part, uint64_t cap,
                                                                      uint32_t* __restrict__ status,
                                                                      const uint32_t* __restrict__ blockhist) {
  extern __shared__ uint32_t sh[];
  uint32_t* hist = sh;            // [H] records per bucket
  uint32_t* loff = sh + H;        // [H] exclusive offsets in the block's sorted order
  uint32_t* gbase = sh + 2 * H;   // [H] first global position of the block's run of each bucket
  uint32_t* cur = sh + 3 * H;     // [H] placement cursors
  uint32_t* s_total = sh + 4 * H;
  uint2* stage = reinterpret_cast<uint2*>(sh + ((4 * H + 1 + 1) & ~1u));  // [2 * kPartEdges]
  uint32_t* gcur = bkt + 2 * H + 1;
  const uint32_t lvl = t.fixed_level >= 0 ? (uint32_t)t.fixed_level : 0u;
  const uint64_t e0 = (uint64_t)blockIdx.x * kPartEdges;
  const uint64_t e1 = min(n, e0 + kPartEdges);
  if (blockhist) {
    // the counts k_part_count took of this same block of edges
    for (uint32_t i = threadIdx.x; i < H; i += blockDim.x) hist[i] = blockhist[(size_t)blockIdx.x * H + i];
  } else {
    for (uint32_t i = threadIdx.x; i < H; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    // out-of-range records were reported by k_part_count; self-loops cancel
    for (uint64_t b = e0; b < e1; b += blockDim.x) {
      const uint64_t e = b + threadIdx.x;
      uint2 p = make_uint2(0, 0);
      if (e < e1) p = pairs[e];
      const bool ok = e < e1 && p.x < t.V && p.y < t.V && p.x != p.y;
      slot_inc(hist, (lvl * t.V + p.x) >> lb, ok);
      slot_inc(hist, (lvl * t.V + p.y) >> lb, ok);
    }
  }
  __syncthreads();
  // exclusive scan of the block histogram: thread i owns buckets [i*per, (i+1)*per)
  {
    const uint32_t per = (H + blockDim.x - 1) / blockDim.x;
    const uint32_t b0 = min(H, threadIdx.x * per), b1 = min(H, b0 + per);
    uint32_t sum = 0;
    for (uint32_t b = b0; b < b1; b++) sum += hist[b];
    uint2 tot;
    const uint2 ex = block_exclusive_scan(make_uint2(sum, 0u), &tot);
    uint32_t run = ex.x;
    for (uint32_t b = b0; b < b1; b++) {
      const uint32_t c = hist[b];
      loff[b] = run;
      cur[b] = run;
      gbase[b] = c ? atomicAdd(&gcur[b], c) : 0u;
      run += c;
    }
    if (threadIdx.x == 0) *s_total = tot.x;
  }
  __syncthreads();
  // every load of the block's edges is issued before the first cursor atomic, so the loads overlap
  for (uint64_t b = e0; b < e1; b += (uint64_t)blockDim.x * kVertUnroll) {
    uint2 ps[kVertUnroll];
#pragma unroll
    for (int j = 0; j < kVertUnroll; j++) {
      const uint64_t e = b + threadIdx.x + (uint64_t)j * blockDim.x;
      ps[j] = e < e1 ? pairs[e] : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int j = 0; j < kVertUnroll; j++) {
      const uint64_t e = b + threadIdx.x + (uint64_t)j * blockDim.x;
      const uint2 p = ps[j];
      const bool ok = e < e1 && p.x < t.V && p.y < t.V && p.x != p.y;
      const uint32_t ku = lvl * t.V + p.x, kv = lvl * t.V + p.y;
      const uint32_t pu = slot_inc(cur, ku >> lb, ok);
      const uint32_t pv = slot_inc(cur, kv >> lb, ok);
      if (ok) {
        stage[pu] = make_uint2(ku, p.y);
        stage[pv] = make_uint2(kv, p.x);
      }
    }
  }
  __syncthreads();
  const uint32_t total = *s_total;
  for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) {
    const uint2 r = stage[i];
    const uint32_t b = r.x >> lb;
    const uint64_t pos = (uint64_t)gbase[b] + (i - loff[b]);
    if (pos >= cap) atomicOr(status, (uint32_t)GS_DEV_ERR_CAPACITY);
    else if (COMPACT) reinterpret_cast<uint32_t*>(part)[pos] = ((r.x & ((1u << lb) - 1u)) << (32u - lb)) | r.y;
    else part[pos] = r;
  }
}

// key within its bucket of pass-1 record i, in either record form
template <bool COMPACT>
__device__ __forceinline__ uint32_t part_key(const uint2* part, uint64_t i, uint32_t lb) {
  if (COMPACT) return reinterpret_cast<const uint32_t*>(part)[i] >> (32u - lb);
  return part[i].x & ((1u << lb) - 1u);
}

// the bucket of pass-2 chunk c: largest d with choff[d] <= c
__device__ __forceinline__ uint32_t chunk_bucket(const uint32_t* choff, uint32_t H, uint32_t c) {
  uint32_t lo = 0, hi = H;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (choff[mid] <= c) lo = mid; else hi = mid;
  }
  return lo;
}

// pass 2, counting: records per vertex of each bucket chunk
// chunkhist (may be null): each chunk's per-vertex counts are also stored at [c << lb], so that the
// sorted placement of the same chunk need not count it again
template <bool COMPACT>
__global__ void __launch_bounds__(kPartThreads) k_vert_count(const uint2* __restrict__ part, const uint32_t* __restrict__ bkt,
                                                             uint32_t H, uint32_t lb, uint32_t* __restrict__ cnt,
                                                             const uint32_t* __restrict__ status,
                                                             uint32_t* __restrict__ chunkhist) {
  extern __shared__ uint32_t hist[];
  __shared__ uint32_t s_d;
  const uint32_t* off = bkt + H;
  const uint32_t* choff = bkt + 3 * H + 1;
  const uint32_t nk = 1u << lb, mask = nk - 1;
  const uint32_t total = status[5];
  for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
    if (threadIdx.x == 0) s_d = chunk_bucket(choff, H, c);
    for (uint32_t i = threadIdx.x; i < nk; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const uint32_t d = s_d;
    const uint32_t r0 = off[d] + (c - choff[d]) * kVertChunk;
    const uint32_t r1 = min(off[d + 1], r0 + kVertChunk);
    for (uint32_t b = r0; b < r1; b += blockDim.x * kVertUnroll) {
      uint32_t ks[kVertUnroll];
#pragma unroll
      for (int j = 0; j < kVertUnroll; j++) {
        const uint32_t i = b + threadIdx.x + j * blockDim.x;
        ks[j] = i < r1 ? part_key<COMPACT>(part, i, lb) : 0xffffffffu;
      }
#pragma unroll
      for (int j = 0; j < kVertUnroll; j++)
        if (ks[j] != 0xffffffffu) atomicAdd(&hist[ks[j]], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nk; k += blockDim.x) {
      if (hist[k]) atomicAdd(&cnt[(d << lb) + k], hist[k]);
      if (chunkhist) chunkhist[((size_t)c << lb) + k] = hist[k];
    }
    __syncthreads();
  }
}

// pass 2, placement: each record's neighbour goes to its vertex's slice of nbr
template <bool COMPACT>
__global__ void __launch_bounds__(kPartThreads) k_vert_scatter(const uint2* __restrict__ part, const uint32_t* __restrict__ bkt,
                                                               uint32_t H, uint32_t lb, uint32_t* __restrict__ cursor,
                                                               uint32_t* __restrict__ nbr, uint64_t cap,
                                                               uint32_t* __restrict__ status) {
  extern __shared__ uint32_t sh[];
  __shared__ uint32_t s_d;
  const uint32_t nk = 1u << lb, mask = nk - 1;
  uint32_t* hist = sh;
  uint32_t* base = sh + nk;
  const uint32_t* off = bkt + H;
  const uint32_t* choff = bkt + 3 * H + 1;
  const uint32_t total = status[5];
  for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
    if (threadIdx.x == 0) s_d = chunk_bucket(choff, H, c);
    for (uint32_t i = threadIdx.x; i < nk; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const uint32_t d = s_d;
    const uint32_t r0 = off[d] + (c - choff[d]) * kVertChunk;
    const uint32_t r1 = min(off[d + 1], r0 + kVertChunk);
    for (uint32_t b = r0; b < r1; b += blockDim.x * kVertUnroll) {
      uint32_t ks[kVertUnroll];
#pragma unroll
      for (int j = 0; j < kVertUnroll; j++) {
        const uint32_t i = b + threadIdx.x + j * blockDim.x;
        ks[j] = i < r1 ? part_key<COMPACT>(part, i, lb) : 0xffffffffu;
      }
#pragma unroll
      for (int j = 0; j < kVertUnroll; j++)
        if (ks[j] != 0xffffffffu) atomicAdd(&hist[ks[j]], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nk; k += blockDim.x) {
      const uint32_t h = hist[k];
      base[k] = h ? atomicAdd(&cursor[(d << lb) + k], h) : 0u;
      hist[k] = 0;
    }
    __syncthreads();
    for (uint32_t b = r0; b < r1; b += blockDim.x * kVertUnroll) {
      uint32_t ks[kVertUnroll], us[kVertUnroll];
#pragma unroll
      for (int j = 0; j < kVertUnroll; j++) {
        const uint32_t i = b + threadIdx.x + j * blockDim.x;
        ks[j] = 0xffffffffu;
        us[j] = 0;
        if (i < r1) {
          if (COMPACT) {
            const uint32_t r = reinterpret_cast<const uint32_t*>(part)[i];
            ks[j] = r >> (32u - lb);
            us[j] = r & ((1u << (32u - lb)) - 1u);
          } else {
            const uint2 r = part[i];
            ks[j] = r.x & mask;
            us[j] = r.y;
          }
        }
      }
#pragma unroll
      for (int j = 0; j < kVertUnroll; j++) {
        if (ks[j] == 0xffffffffu) continue;
        const uint32_t pos = base[ks[j]] + atomicAdd(&hist[ks[j]], 1u);
        if (pos < cap) nbr[pos] = us[j];
        else atomicOr(&status[0], (uint32_t)GS_DEV_ERR_CAPACITY);
      }
    }
    __syncthreads();
  }
}

// pass 2, placement with one-word records, sorted in shared memory: a block loads its chunk once
// (kVertChunk / kPartThreads records per thread, held in registers), counts them per vertex, reserves
// each vertex's run in the output, sorts the chunk by vertex into a shared stage (the record keeps its
// bucket-local key in its top bits), and writes the stage out with consecutive threads on consecutive
// addresses of each vertex's run.  The scattered one-record stores of k_vert_scatter cost one L2 sector
// request per record; these cost one per 32 bytes of a run.
constexpr int kVertPer = kVertChunk / kPartThreads;   // records per thread per chunk
static_assert(kVertPer * kPartThreads == kVertChunk, "a chunk is a whole number of records per thread");

size_t vert_scatter_sorted_smem(uint32_t lb) {
  return (size_t)4 * (1u << lb) * sizeof(uint32_t) + (size_t)kVertChunk * sizeof(uint32_t);
}

// three blocks per SM (at most 42 registers a thread): the chunk's records wait in registers while the
// block scans, and a third resident block keeps loads in flight meanwhile
__global__ void __launch_bounds__(kPartThreads, 3) k_vert_scatter_sorted(const uint32_t* __restrict__ part,
                                                                      const uint32_t* __restrict__ bkt, uint32_t H,
                                                                      uint32_t lb, uint32_t* __restrict__ cursor,
                                                                      uint32_t* __restrict__ nbr, uint64_t cap,
                                                                      uint32_t* __restrict__ status,
                                                                      const uint32_t* __restrict__ chunkhist) {
  extern __shared__ uint32_t sh[];
  __shared__ uint32_t s_d;
  const uint32_t nk = 1u << lb;
  uint32_t* hist = sh;            // [nk] records per vertex of the chunk
  uint32_t* loff = sh + nk;       // [nk] first stage slot of each vertex
  uint32_t* base = sh + 2 * nk;   // [nk] first output position of each vertex's run
  uint32_t* cur = sh + 3 * nk;    // [nk] stage cursors
  uint32_t* stage = sh + 4 * nk;  // [kVertChunk] records sorted by vertex
  const uint32_t* off = bkt + H;
  const uint32_t* choff = bkt + 3 * H + 1;
  const uint32_t shift = 32u - lb, umask = (1u << shift) - 1u;
  const uint32_t total = status[5];
  for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
    if (threadIdx.x == 0) s_d = chunk_bucket(choff, H, c);
    if (chunkhist) {
      // the counts k_vert_count took of this same chunk
      for (uint32_t i = threadIdx.x; i < nk; i += blockDim.x) hist[i] = chunkhist[((size_t)c << lb) + i];
    } else {
      for (uint32_t i = threadIdx.x; i < nk; i += blockDim.x) hist[i] = 0;
    }
    __syncthreads();
    const uint32_t d = s_d;
    const uint32_t r0 = off[d] + (c - choff[d]) * kVertChunk;
    const uint32_t r1 = min(off[d + 1], r0 + kVertChunk);
    uint32_t rec[kVertPer];
#pragma unroll
    for (int j = 0; j < kVertPer; j++) {
      const uint32_t i = r0 + threadIdx.x + j * blockDim.x;
      rec[j] = i < r1 ? part[i] : 0xffffffffu;
    }
    if (!chunkhist) {
#pragma unroll
      for (int j = 0; j < kVertPer; j++)
        if (r0 + threadIdx.x + j * blockDim.x < r1) atomicAdd(&hist[rec[j] >> shift], 1u);
    }
    __syncthreads();
    // block scan of the counts (thread t owns vertices [t*per, (t+1)*per)) and the global reservations
    {
      const uint32_t per = (nk + blockDim.x - 1) / blockDim.x;
      const uint32_t k0 = min(nk, threadIdx.x * per), k1 = min(nk, k0 + per);
      uint32_t sum = 0;
      for (uint32_t k = k0; k < k1; k++) sum += hist[k];
      uint2 tot;
      uint32_t run = block_exclusive_scan(make_uint2(sum, 0u), &tot).x;
      for (uint32_t k = k0; k < k1; k++) {
        const uint32_t h = hist[k];
        loff[k] = run;
        cur[k] = run;
        base[k] = h ? atomicAdd(&cursor[(d << lb) + k], h) : 0u;
        run += h;
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kVertPer; j++)
      if (r0 + threadIdx.x + j * blockDim.x < r1) stage[atomicAdd(&cur[rec[j] >> shift], 1u)] = rec[j];
    __syncthreads();
    const uint32_t n = r1 - r0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t r = stage[i];
      const uint32_t k = r >> shift;
      const uint32_t pos = base[k] + (i - loff[k]);
      if (pos < cap) nbr[pos] = r & umask;
      else atomicOr(&status[0], (uint32_t)GS_DEV_ERR_CAPACITY);
    }
    __syncthreads();
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
    status[14] = 0;  // next work chunk of the packed sketch update
  }
}

// adds the tile prefixes and resets the counters to the record cursors used by the scatter; with an
// owner table, also records the vertex of each of its work chunks below owner_cap, so the sketch
// update finds a chunk's vertex with one load instead of a search over choff
__global__ void __launch_bounds__(kScanThreads) k_scan_add(uint32_t* __restrict__ off, uint32_t* __restrict__ choff,
                                                           uint32_t* __restrict__ cursor,
                                                           const uint32_t* __restrict__ tile_sums, uint32_t nv,
                                                           uint32_t chunk, uint32_t* __restrict__ owner,
                                                           uint32_t owner_cap) {
  const uint32_t t = blockIdx.x;
  const uint32_t a = tile_sums[2 * t], b = tile_sums[2 * t + 1];
  const uint64_t base = (uint64_t)t * kScanTile + (uint64_t)threadIdx.x * kScanPer;
  const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    const uint64_t i = base + k;
    uint32_t c0 = 0, n = 0;
    if (i < nv) {
      const uint32_t o = off[i] + a;
      off[i] = o;
      c0 = choff[i] + b;
      choff[i] = c0;
      if (owner) n = (cursor[i] + chunk - 1) / chunk;   // cursor still holds the count here
      cursor[i] = o;
    }
    if (owner) {
      // a vertex of a few chunks writes its own entries; the warp writes a hub vertex's together
      constexpr uint32_t kOwnFew = 8;
      if (n <= kOwnFew)
        for (uint32_t c = c0; c < c0 + n && c < owner_cap; c++) owner[c] = (uint32_t)i;
      for (uint32_t m = __ballot_sync(0xffffffffu, n > kOwnFew); m; m &= m - 1) {
        const uint32_t src = __ffs(m) - 1;
        const uint32_t hc0 = __shfl_sync(0xffffffffu, c0, src), hn = __shfl_sync(0xffffffffu, n, src);
        const uint32_t hv = __shfl_sync(0xffffffffu, (uint32_t)i, src);
        for (uint32_t c = hc0 + lane; c < hc0 + hn && c < owner_cap; c += 32) owner[c] = hv;
      }
    }
  }
}

// ---- the sketch update ----

struct IngestArgs {
  const uint32_t* off;
  const uint32_t* choff;
  const uint32_t* nbr;
  GsBucket* sk;
  const uint64_t* colmix;   // [C] column constants, [C] = checksum constant; per tenant: [T][kColStride]
  const uint32_t* status;   // [2] = work chunks
  uint32_t nv, V, C, bkt, nb, chunk;
  const uint32_t* vtenant;       // tenant of every vertex (tenant variant only)
  const GsIngTenant* tenants;    // geometry and arena offset of every tenant (tenant variant only)
  uint32_t warp_words;           // shared memory per warp in uint4 (packed variant only)
  uint32_t* next_chunk;          // work-chunk counter, zero at launch (packed variant only)
  const uint32_t* owner;         // vertex of every work chunk below owner_cap (may be null)
  uint32_t owner_cap;
};

// ---- packed lane layout (sketches of at most 24 columns) ----
//
// With one column per lane, a sketch of C < 32 columns leaves 32 - C lanes idle on every record
// (8 of 32 at V = 2^17).  The packed layout covers the C columns of four records with 32 lanes in
// kPackRounds = 3 steps.  With se = ceil(C / 3) <= 8 and the columns cut into three blocks of se,
// lane s se + i (slot s < 4, i < se) holds record s of the group for all three steps, and in step j
//   * a main slot s < 3 takes column i + se ((j + s) mod 3) of its record: in every step the three
//     main slots cover the three column blocks, so the main lanes touch distinct columns;
//   * the spare slot s = 3 takes column i + j se of record 3.
// (nothing when the column is >= C).  A full batch of 32 staged records takes 24 steps instead of 32
// at C = 24, and a lane loads its record once per group: a 16-byte load costs the same four shared-
// memory wavefronts whether 8 or 32 lanes share its address, and with the update's read and write of
// a 16-byte row those wavefronts are the kernel's bound.  Column, column constant and row block of
// every (lane, step) are fixed per geometry and held in registers.  Column c keeps main rows
// [depth][c] (pitch p1 = C rounded up to 8) whichever main lane updates it in a step, so the steps are
// separated by __syncwarp; spare lane 3 se + i keeps its own rows [j][depth][lane % 8] (pitch 8; se <=
// 8, so the spare lanes' residues are distinct).  A lane's entry sits at its column (main) or lane
// (spare) mod 8, so a quarter-warp's accesses stay in distinct bank groups whatever depths its lanes
// hit.  At the end of a chunk column c gathers its main row and the rows of spare lane 3 se + c % se,
// step c / se.  Records left over after the groups of four (and every record of a wider sketch) take
// one step each on lanes c < C, lane c taking column c.
constexpr uint32_t kPackRounds = 3;
constexpr uint32_t kPackMaxCols = 24;  // ceil(C / 3) <= 32 - C
constexpr uint32_t kRecWords = 32;
// rows per lane block: depths 0..kSlabDepth-1 and one discard row, which takes the XOR of every
// (record, column) that has no row (deeper buckets, spare rounds without a column) so that the hot
// loop updates a row unconditionally; the discard row is never merged
constexpr uint32_t kPackRowsAlloc = kSlabDepth + 1;
// at most 12 warps per block, two blocks per SM: with 8 KB of rows per warp shared memory holds 24
// warps per SM, and the register cap that two 384-thread blocks leave (85) avoids spills
constexpr int kPackMaxThreads = 384;

GS_HD uint32_t pack_spare_lanes(uint32_t C) { return C <= kPackMaxCols ? (C + kPackRounds - 1) / kPackRounds : 0u; }
GS_HD uint32_t pack_p1(uint32_t C) { return (C + 7u) & ~7u; }

// uint4 words per warp: rows of the main lanes and of the spare slots, then the staged records
GS_HD uint32_t pack_warp_words(uint32_t C) {
  return (uint32_t)kPackRowsAlloc * (pack_p1(C) + (pack_spare_lanes(C) ? kPackRounds * 8u : 0u)) + kRecWords;
}

__device__ __forceinline__ uint32_t chunk_owner(const IngestArgs& A, uint32_t ch, uint32_t lane) {
  uint32_t lo = 0, hi = A.nv;
  while (hi - lo > 1) {
    const uint32_t step = (hi - lo + 31) / 32;
    const uint32_t probe = lo + (lane + 1) * step;
    const bool le = probe < hi && A.choff[probe] <= ch;
    const uint32_t k = __popc(__ballot_sync(0xffffffffu, le));
    lo = lo + k * step;
    hi = min(hi, lo + step);
  }
  return lo;
}

__device__ __forceinline__ void xor_bucket_global(GsBucket* p, uint64_t a, uint64_t g) {
  atomicXor(reinterpret_cast<unsigned long long*>(&p->alpha), (unsigned long long)a);
  atomicXor(reinterpret_cast<unsigned long long*>(&p->gamma), (unsigned long long)g);
}

// XOR one record {mix(k'), checksum} = q into bucket depth d of column c: registers for d < R, the
// lane's shared-memory row for d < kSlabDepth, HBM beyond; d == bkt (or c >= C) touches nothing.
template <int R, bool SMALL>
__device__ __forceinline__ void apply_update(uint4* acc, uint4* slab_g, GsBucket* skv, uint32_t c, uint32_t C,
                                             uint32_t bkt, uint32_t d, const uint4& q) {
  constexpr int kRows = kSlabDepth - R;
  const bool live = c < C;
#pragma unroll
  for (int k = 0; k < R; k++) {
    const bool hit = live && d == (uint32_t)k && (!SMALL || d < bkt);
    if (hit) { acc[k].x ^= q.x; acc[k].y ^= q.y; acc[k].z ^= q.z; acc[k].w ^= q.w; }
  }
  if (live && d >= (uint32_t)R && (!SMALL || d < bkt)) {
    if (d < (uint32_t)kSlabDepth) {
      uint4* p = slab_g + (d - R) * kSlabPitch + (c & 31u);
      uint4 t = *p;
      t.x ^= q.x; t.y ^= q.y; t.z ^= q.z; t.w ^= q.w;
      *p = t;
    } else if (d < bkt) {
      xor_bucket_global(skv + (size_t)c * bkt + d, gs_key_unmix(((uint64_t)q.y << 32) | q.x),
                        ((uint64_t)q.w << 32) | q.z);
    }
  }
  (void)kRows;
}

// Per lane: buckets of depth < kRegDepth of its column(s) in registers, depth [kRegDepth, kSlabDepth)
// in a lane-private shared-memory row, deeper ones straight into HBM.  Buckets accumulate
// {mix(k'), checksum} instead of {edge id, checksum}: gs_key_mix is XOR-linear, so XOR-ing mixed
// keys and unmixing once per bucket at merge time (gs_key_unmix) gives the XOR of the edge ids, and
// every record is a single 16-byte broadcast {mix(k'), checksum}.
// R: depths held in registers.  SMALL: the geometry has bkt_per_col < kSlabDepth (V <= 23), so every
// path checks the depth against bkt_per_col; otherwise only the rare global path does.
// TEN: the vertices belong to independent graphs of an engine; each work chunk looks up its tenant's
// geometry, column constants and arena offset.
template <int CG, int R, bool SMALL, bool TEN>
__global__ void __launch_bounds__(512) k_ingest(const IngestArgs A) {
  extern __shared__ uint4 smem[];
  constexpr int kRegDepth = R;
  constexpr int kRows = kSlabDepth - kRegDepth;
  constexpr int kSlabWords = CG * kRows * kSlabPitch;  // uint4 per warp slab
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  uint4* slab = smem + (size_t)wib * (kSlabWords + 32);
  uint4* rec = slab + kSlabWords;                     // 32 x {mix(k'), checksum}

  uint32_t C = A.C, bkt = A.bkt, nb = A.nb;
  const uint32_t V = A.V;
  uint64_t csmix = 0;
  uint64_t cmix[CG];
  uint32_t cur_t = 0xffffffffu;
  if (!TEN) {
    csmix = A.colmix[C];
#pragma unroll
    for (int g = 0; g < CG; g++) {
      const uint32_t c = lane + 32u * g;
      cmix[g] = c < C ? A.colmix[c] : 0ull;
    }
  }

  const uint32_t total = A.status[2];
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;

  // with a chunk counter, warps take work chunks from it (lane 0 fetches the next index while the
  // current chunk runs); without one, a fixed stride
  const bool dyn = A.next_chunk != nullptr;
  uint32_t nxt = 0;
  if (dyn && lane == 0) nxt = atomicAdd(A.next_chunk, 1u);
  for (uint32_t ch = dyn ? __shfl_sync(0xffffffffu, nxt, 0) : gw; ch < total;
       ch = dyn ? __shfl_sync(0xffffffffu, nxt, 0) : ch + nw) {
    if (dyn && lane == 0) nxt = atomicAdd(A.next_chunk, 1u);
    const uint32_t vv = ch < A.owner_cap ? A.owner[ch] : chunk_owner(A, ch, lane);
    const uint32_t c0 = A.choff[vv];
    // a vertex of one chunk is this warp's alone: its merge is a plain read-modify-write (many small
    // vertices, as an engine's tenants have, would saturate the L2 atomics)
    const bool exclusive = (A.choff[vv + 1] - c0) == 1;
    const uint32_t rb = A.off[vv] + (ch - c0) * A.chunk;
    const uint32_t re = min(A.off[vv + 1], rb + A.chunk);
    uint32_t v, vb = 0;  // vb: first engine vertex id of the tenant (neighbours are stored engine-wide)
    GsBucket* skv;
    if (TEN) {
      const uint32_t t = A.vtenant[vv];
      const GsIngTenant T = A.tenants[t];
      if (t != cur_t) {
        cur_t = t;
        C = T.C;
        bkt = T.bkt;
        nb = T.nb;
        const uint64_t* cm = A.colmix + (size_t)t * kColStride;
        csmix = cm[C];
#pragma unroll
        for (int g = 0; g < CG; g++) {
          const uint32_t c = lane + 32u * g;
          cmix[g] = c < C ? cm[c] : 0ull;
        }
      }
      vb = T.vbase;
      v = vv - vb;
      skv = A.sk + T.sk_off + (size_t)v * nb;
    } else {
      v = vv % V;
      skv = A.sk + (size_t)vv * nb;
    }

    for (int i = lane; i < kSlabWords; i += 32) slab[i] = make_uint4(0, 0, 0, 0);
    uint4 acc[CG][kRegDepth > 0 ? kRegDepth : 1];
#pragma unroll
    for (int g = 0; g < CG; g++)
#pragma unroll
      for (int d = 0; d < kRegDepth; d++) acc[g][d] = make_uint4(0, 0, 0, 0);
    uint64_t det_m = 0, det_g = 0;
    __syncwarp();

    for (uint32_t b = rb; b < re; b += 32) {
      const uint32_t r = b + lane;
      const bool valid = r < re;
      const uint32_t u = valid ? A.nbr[r] - vb : v;
      const uint64_t E = gs_key_mix(gs_concat(v, u));
      const uint64_t cs = gs_hash_tail(E ^ csmix);
      if (valid) { det_m ^= E; det_g ^= cs; }
      rec[lane] = make_uint4((uint32_t)E, (uint32_t)(E >> 32), (uint32_t)cs, (uint32_t)(cs >> 32));
      __syncwarp();
      const uint32_t cnt = min(32u, re - b);
      // four (then two, then one) records per iteration: their hash chains are independent and
      // overlap in the pipeline
      uint32_t j = 0;
      for (; j + 3 < cnt; j += 4) {
        const uint4 q0 = rec[j], q1 = rec[j + 1], q2 = rec[j + 2], q3 = rec[j + 3];
        const uint64_t E0 = ((uint64_t)q0.y << 32) | q0.x, E1 = ((uint64_t)q1.y << 32) | q1.x;
        const uint64_t E2 = ((uint64_t)q2.y << 32) | q2.x, E3 = ((uint64_t)q3.y << 32) | q3.x;
#pragma unroll
        for (int g = 0; g < CG; g++) {
          const uint32_t d0 = gs_depth_from_mixed(E0 ^ cmix[g], bkt);
          const uint32_t d1 = gs_depth_from_mixed(E1 ^ cmix[g], bkt);
          const uint32_t d2 = gs_depth_from_mixed(E2 ^ cmix[g], bkt);
          const uint32_t d3 = gs_depth_from_mixed(E3 ^ cmix[g], bkt);
          apply_update<R, SMALL>(acc[g], slab + g * kRows * kSlabPitch, skv, lane + 32u * g, C, bkt, d0, q0);
          apply_update<R, SMALL>(acc[g], slab + g * kRows * kSlabPitch, skv, lane + 32u * g, C, bkt, d1, q1);
          apply_update<R, SMALL>(acc[g], slab + g * kRows * kSlabPitch, skv, lane + 32u * g, C, bkt, d2, q2);
          apply_update<R, SMALL>(acc[g], slab + g * kRows * kSlabPitch, skv, lane + 32u * g, C, bkt, d3, q3);
        }
      }
      for (; j + 1 < cnt; j += 2) {
        const uint4 q0 = rec[j], q1 = rec[j + 1];
        const uint64_t E0 = ((uint64_t)q0.y << 32) | q0.x, E1 = ((uint64_t)q1.y << 32) | q1.x;
#pragma unroll
        for (int g = 0; g < CG; g++) {
          const uint32_t d0 = gs_depth_from_mixed(E0 ^ cmix[g], bkt);
          const uint32_t d1 = gs_depth_from_mixed(E1 ^ cmix[g], bkt);
          apply_update<R, SMALL>(acc[g], slab + g * kRows * kSlabPitch, skv, lane + 32u * g, C, bkt, d0, q0);
          apply_update<R, SMALL>(acc[g], slab + g * kRows * kSlabPitch, skv, lane + 32u * g, C, bkt, d1, q1);
        }
      }
      if (j < cnt) {
        const uint4 q0 = rec[j];
        const uint64_t E0 = ((uint64_t)q0.y << 32) | q0.x;
#pragma unroll
        for (int g = 0; g < CG; g++) {
          const uint32_t d0 = gs_depth_from_mixed(E0 ^ cmix[g], bkt);
          apply_update<R, SMALL>(acc[g], slab + g * kRows * kSlabPitch, skv, lane + 32u * g, C, bkt, d0, q0);
        }
      }
      __syncwarp();
    }

    // merge the register depths: lane c owns the first kRegDepth buckets of column c
#pragma unroll
    for (int g = 0; g < CG; g++) {
      const uint32_t c = lane + 32u * g;
      if (c >= C) continue;
#pragma unroll
      for (int d = 0; d < kRegDepth; d++) {
        const uint4 t = acc[g][d];
        if ((uint32_t)d >= bkt || (t.x | t.y | t.z | t.w) == 0u) continue;
        const uint64_t a = gs_key_unmix(((uint64_t)t.y << 32) | t.x), gm = ((uint64_t)t.w << 32) | t.z;
        GsBucket* p = skv + (size_t)c * bkt + d;
        if (exclusive) { p->alpha ^= a; p->gamma ^= gm; }
        else xor_bucket_global(p, a, gm);
      }
    }
    __syncwarp();
    // merge the slab rows: item i -> column i / kRows, depth kRegDepth + i % kRows, so consecutive lanes
    // cover contiguous buckets of one column
#pragma unroll
    for (int g = 0; g < CG; g++) {
      const uint32_t cols = min(32u, C - min(C, 32u * g));
      for (uint32_t i = lane; i < cols * kRows; i += 32) {
        const uint32_t cl = i / kRows, row = i % kRows;
        const uint4 t = slab[(g * kRows + row) * kSlabPitch + cl];
        if (kRegDepth + row >= bkt || (t.x | t.y | t.z | t.w) == 0u) continue;
        const uint64_t a = gs_key_unmix(((uint64_t)t.y << 32) | t.x), gm = ((uint64_t)t.w << 32) | t.z;
        GsBucket* p = skv + (size_t)(cl + 32u * g) * bkt + kRegDepth + row;
        if (exclusive) { p->alpha ^= a; p->gamma ^= gm; }
        else xor_bucket_global(p, a, gm);
      }
    }
    // deterministic bucket (last bucket of the sketch)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      det_m ^= __shfl_xor_sync(0xffffffffu, det_m, o);
      det_g ^= __shfl_xor_sync(0xffffffffu, det_g, o);
    }
    if (lane == 0 && (det_m | det_g) != 0ull) {
      GsBucket* p = skv + (nb - 1);
      const uint64_t a = gs_key_unmix(det_m);
      if (exclusive) { p->alpha ^= a; p->gamma ^= det_g; }
      else xor_bucket_global(p, a, det_g);
    }
    __syncwarp();
  }
}

// Sketch update with the packed lane layout (reg_depth 0, at most 32 columns); chunk lookup, record
// staging, deep-bucket path and merge as in k_ingest.
template <bool TEN>
__global__ void __launch_bounds__(kPackMaxThreads, 2) k_ingest_packed(const IngestArgs A) {
  extern __shared__ uint4 smem[];
  constexpr uint32_t kRows = kSlabDepth;
  constexpr uint32_t kRA = kPackRowsAlloc;
  constexpr uint32_t J = kPackRounds;
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  uint4* const wbase = smem + (size_t)wib * A.warp_words;
  uint4* const rec = wbase + A.warp_words - kRecWords;

  uint32_t C = 0, bkt = A.bkt, nb = A.nb, se = 0, p1 = 8;
  const uint32_t V = A.V;
  uint64_t csmix = 0, cmix = 0;
  // per lane: record slot of a group and, per step, column (>= C: none), column constant, row block
  uint32_t ro = 0, sb[J], col[J], pitch = 0, msp = 0;
  uint64_t cm[J];
  auto set_geometry = [&](uint32_t c_new, const uint64_t* cmt) {
    C = c_new;
    se = pack_spare_lanes(C);
    p1 = pack_p1(C);
    csmix = cmt[C];
    cmix = lane < C ? cmt[lane] : 0ull;
    // slot (J + 1: no record of the groups, also every lane of a wider sketch) and index in the slot
    const uint32_t sl = se ? min(lane / se, J + 1) : J + 1, i = se ? lane % se : 0u;
    ro = min(sl, J);
    pitch = sl < J ? p1 : 8u;
    // the merge's lane c < C: word of column c's spare rows (spare lane J se + c % se, step c / se)
    msp = se && lane < C ? kRA * p1 + (lane / se) * kRA * 8u + ((J * se + lane % se) & 7u) : 0u;
#pragma unroll
    for (uint32_t j = 0; j < J; j++) {
      const uint32_t c = sl < J ? i + se * ((j + sl) % J) : (sl == J ? i + se * j : 0xffffffffu);
      col[j] = c < C ? c : 0xffffffffu;
      cm[j] = c < C ? cmt[c] : 0ull;
      // a main lane without a column uses the discard row of column i
      sb[j] = sl < J ? (c < C ? c : i) : kRA * p1 + (j * kRA) * 8u + (lane & 7u);
    }
  };
  uint32_t cur_t = 0xffffffffu;
  if (!TEN) set_geometry(A.C, A.colmix);

  const uint32_t total = A.status[2];
  // warps take work chunks from a counter, so no warp idles while others still have long chunks
  // left; lane 0 fetches the next index while the current chunk runs
  uint32_t nxt = 0;
  if (lane == 0) nxt = atomicAdd(A.next_chunk, 1u);
  for (uint32_t ch = __shfl_sync(0xffffffffu, nxt, 0); ch < total; ch = __shfl_sync(0xffffffffu, nxt, 0)) {
    if (lane == 0) nxt = atomicAdd(A.next_chunk, 1u);
    const uint32_t vv = ch < A.owner_cap ? A.owner[ch] : chunk_owner(A, ch, lane);
    const uint32_t c0ff = A.choff[vv];
    const uint32_t rb = A.off[vv] + (ch - c0ff) * A.chunk;
    const uint32_t re = min(A.off[vv + 1], rb + A.chunk);
    uint32_t v, vb = 0;
    GsBucket* skv;
    if (TEN) {
      const uint32_t t = A.vtenant[vv];
      const GsIngTenant T = A.tenants[t];
      if (t != cur_t) {
        cur_t = t;
        bkt = T.bkt;
        nb = T.nb;
        set_geometry(T.C, A.colmix + (size_t)t * kColStride);
      }
      vb = T.vbase;
      v = vv - vb;
      skv = A.sk + T.sk_off + (size_t)v * nb;
    } else {
      v = vv % V;
      skv = A.sk + (size_t)vv * nb;
    }

    const uint32_t zw = kRA * (p1 + (se ? J * 8u : 0u));
    // every lane with a column in every step (C = 24): no per-step lane test
    const bool all_live = C + se == 32u && J * se == C;
    for (uint32_t i = lane; i < zw; i += 32) wbase[i] = make_uint4(0, 0, 0, 0);
    uint64_t det_m = 0, det_g = 0;
    __syncwarp();

    // 32-bit shared-window addresses: row block bb of this warp at ws + 16 bb, record k at rs + 16 k
    const uint32_t ws = (uint32_t)__cvta_generic_to_shared(wbase);
    const uint32_t rs = (uint32_t)__cvta_generic_to_shared(rec);
    const uint32_t pitch16 = pitch * 16u, p116 = p1 * 16u;
    // cap = min(bkt_per_col, kRows): depths below it are buckets held in the lane's rows, and row cap
    // is the discard row (depth kRows, or bkt_per_col = no bucket).  Only a geometry with more
    // buckets per column than rows has buckets deeper than the rows (the rare HBM path).  The cap is
    // taken per work chunk: the tenants of one engine launch can have either kind of geometry.
    const uint32_t cap = min(bkt, kRows);
    const uint32_t capbit = 1u << cap;
    // XOR record q into the lane's column cc at the depth whose low-word part is dl (gs_depth_low;
    // high product word h2), rows at row block bb.  Depths below cap go to the lane's rows; a depth of
    // kRows or more is completed from the high word (also when the low word was zero) and, when it is
    // below bkt_per_col, goes to HBM; anything else has no bucket.
    auto update = [&](bool live, uint32_t bb, uint32_t cc, uint32_t dl, uint32_t h2, const uint4& q) {
      if (live && dl < cap) {
        const uint32_t a = ws + bb * 16u + dl * p116;
        uint4 t;
        asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(t.x), "=r"(t.y), "=r"(t.z), "=r"(t.w) : "r"(a));
        t.x ^= q.x; t.y ^= q.y; t.z ^= q.z; t.w ^= q.w;
        asm volatile("st.shared.v4.u32 [%0], {%1,%2,%3,%4};" :: "r"(a), "r"(t.x), "r"(t.y), "r"(t.z), "r"(t.w)
                     : "memory");
      } else if (live && dl >= kRows) {
        const uint32_t dd = gs_depth_finish(dl, h2, bkt);
        if (dd < bkt)
          xor_bucket_global(skv + (size_t)cc * bkt + dd, gs_key_unmix(((uint64_t)q.y << 32) | q.x),
                            ((uint64_t)q.w << 32) | q.z);
      }
    };
    // The groups' row update, branch-free: the depth comes capped at `cap` (gs_depth_capped), and
    // rounds without a column use `cap` as well.  A lane whose depth reached kRows (possible only
    // when bkt_per_col >= kRows) completes it from the full hash on the rare HBM path (`deep`) after
    // the group.
    auto rowx = [&](uint32_t bb, uint32_t d, const uint4& q) {
      const uint32_t a = ws + bb * 16u + d * pitch16;
      uint4 t;
      asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(t.x), "=r"(t.y), "=r"(t.z), "=r"(t.w) : "r"(a));
      t.x ^= q.x; t.y ^= q.y; t.z ^= q.z; t.w ^= q.w;
      asm volatile("st.shared.v4.u32 [%0], {%1,%2,%3,%4};" :: "r"(a), "r"(t.x), "r"(t.y), "r"(t.z), "r"(t.w)
                   : "memory");
    };
    auto deep = [&](bool live, uint32_t cc, uint32_t dl, uint64_t cmj, const uint4& q) {
      if (live && dl >= kRows) {
        const uint32_t dd = gs_depth_from_mixed((((uint64_t)q.y << 32) | q.x) ^ cmj, bkt);
        if (dd < bkt)
          xor_bucket_global(skv + (size_t)cc * bkt + dd, gs_key_unmix(((uint64_t)q.y << 32) | q.x),
                            ((uint64_t)q.w << 32) | q.z);
      }
    };
    auto lds = [](uint32_t a) {
      uint4 q;
      asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(q.x), "=r"(q.y), "=r"(q.z), "=r"(q.w) : "r"(a));
      return q;
    };
    auto emix = [](const uint4& q) { return ((uint64_t)q.y << 32) | q.x; };

    // each batch's neighbour ids are loaded one batch ahead, so the load overlaps the previous rounds
    uint32_t nxt = rb + lane < re ? A.nbr[rb + lane] : 0u;
    for (uint32_t b = rb; b < re; b += 32) {
      const uint32_t r = b + lane;
      const bool valid = r < re;
      const uint32_t u = valid ? nxt - vb : v;
      if (r + 32 < re) nxt = A.nbr[r + 32];
      const uint64_t E = gs_key_mix(gs_concat(v, u));
      const uint64_t cs = gs_hash_tail(E ^ csmix);
      if (valid) { det_m ^= E; det_g ^= cs; }
      rec[lane] = make_uint4((uint32_t)E, (uint32_t)(E >> 32), (uint32_t)cs, (uint32_t)(cs >> 32));
      __syncwarp();
      const uint32_t cnt = min(32u, re - b);
      const uint32_t ng = se ? cnt >> 2 : 0u;
      uint32_t k = 0;
      // groups of four records; ar: this lane's record of the group.  A main column's rows pass to
      // another lane from one step to the next, hence the __syncwarp after every step.
      uint32_t ar = rs + ro * 16u;
      uint32_t gi = 0;
      if (all_live) {
#pragma unroll 2
        for (; gi < ng; gi++, k += J + 1, ar += 16u * (J + 1)) {
          const uint4 q = lds(ar);
          const uint64_t e = emix(q);
          const uint32_t d0 = gs_depth_capped(e ^ cm[0], capbit);
          const uint32_t d1 = gs_depth_capped(e ^ cm[1], capbit);
          const uint32_t d2 = gs_depth_capped(e ^ cm[2], capbit);
          rowx(sb[0], d0, q);
          __syncwarp();
          rowx(sb[1], d1, q);
          __syncwarp();
          rowx(sb[2], d2, q);
          __syncwarp();
          if (max(d0, max(d1, d2)) >= kRows) {
            deep(true, col[0], d0, cm[0], q);
            deep(true, col[1], d1, cm[1], q);
            deep(true, col[2], d2, cm[2], q);
          }
        }
      }
      for (; gi < ng; gi++, k += J + 1, ar += 16u * (J + 1)) {
        const uint4 q = lds(ar);
        const uint64_t e = emix(q);
        const uint32_t d0 = gs_depth_capped(e ^ cm[0], capbit);
        const uint32_t d1 = gs_depth_capped(e ^ cm[1], capbit);
        const uint32_t d2 = gs_depth_capped(e ^ cm[2], capbit);
        const bool l0 = col[0] < C, l1 = col[1] < C, l2 = col[2] < C;
        rowx(sb[0], l0 ? d0 : cap, q);
        __syncwarp();
        rowx(sb[1], l1 ? d1 : cap, q);
        __syncwarp();
        rowx(sb[2], l2 ? d2 : cap, q);
        __syncwarp();
        if (max(d0, max(d1, d2)) >= kRows) {
          deep(l0, col[0], d0, cm[0], q);
          deep(l1, col[1], d1, cm[1], q);
          deep(l2, col[2], d2, cm[2], q);
        }
      }
      // the rest: one record per step on lanes c < C
      const bool main = lane < C;
      for (; k + 1 < cnt; k += 2) {
        const uint4 q0 = lds(rs + 16u * k), q1 = lds(rs + 16u * (k + 1));
        uint32_t h0, h1;
        const uint32_t d0 = gs_depth_low(emix(q0) ^ cmix, &h0);
        const uint32_t d1 = gs_depth_low(emix(q1) ^ cmix, &h1);
        update(main, lane, lane, d0, h0, q0);
        update(main, lane, lane, d1, h1, q1);
      }
      if (k < cnt) {
        const uint4 q0 = lds(rs + 16u * k);
        uint32_t h0;
        const uint32_t d0 = gs_depth_low(emix(q0) ^ cmix, &h0);
        update(main, lane, lane, d0, h0, q0);
      }
      __syncwarp();
    }

    // merge: one depth at a time, lane c on column c, so a quarter-warp reads eight columns of one
    // row (eight bank groups); a column's spare rows (if any) are folded in first
    if (lane < C) {
      for (uint32_t row = 0; row < cap; row++) {
        uint4 t = wbase[row * p1 + lane];
        if (se) {
          const uint4 t2 = wbase[msp + row * 8u];
          t.x ^= t2.x; t.y ^= t2.y; t.z ^= t2.z; t.w ^= t2.w;
        }
        if ((t.x | t.y | t.z | t.w) == 0u) continue;
        const uint64_t a = gs_key_unmix(((uint64_t)t.y << 32) | t.x), gm = ((uint64_t)t.w << 32) | t.z;
        GsBucket* p = skv + (size_t)lane * bkt + row;
        xor_bucket_global(p, a, gm);
      }
    }
    // deterministic bucket (last bucket of the sketch)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      det_m ^= __shfl_xor_sync(0xffffffffu, det_m, o);
      det_g ^= __shfl_xor_sync(0xffffffffu, det_g, o);
    }
    if (lane == 0 && (det_m | det_g) != 0ull) {
      GsBucket* p = skv + (nb - 1);
      const uint64_t a = gs_key_unmix(det_m);
      xor_bucket_global(p, a, det_g);
    }
    __syncwarp();
  }
}

size_t ingest_smem_bytes(int cg, int r, int warps) {
  return (size_t)warps * (size_t)(cg * (kSlabDepth - r) * kSlabPitch + 32) * sizeof(uint4);
}

template <int CG, int R, bool SMALL, bool TEN>
gs_status launch_ingest(gs_graph* g, uint32_t nv, cudaStream_t s) {
  IngestArgs A;
  A.off = g->d_off; A.choff = g->d_choff; A.nbr = g->d_nbr; A.sk = g->d_sk; A.colmix = g->d_colmix;
  A.status = g->d_status; A.nv = nv; A.V = g->V; A.C = g->geom.num_columns;
  A.bkt = g->geom.bkt_per_col; A.nb = g->geom.num_buckets; A.chunk = g->tune.chunk;
  A.warp_words = 0;
  A.next_chunk = g->d_status + 14;
  A.owner = g->d_owner;
  A.owner_cap = (uint32_t)g->owner_cap;
  const int warps = (int)g->tune.warps_per_block;
  const size_t smem = ingest_smem_bytes(CG, R, warps);
  // the opt-in shared-memory limit is a per-device function attribute; the persistent grid fills
  // every SM with as many blocks as registers and shared memory allow
  struct Cache { size_t smem = 0; int warps = 0; int blocks = 0; };
  static thread_local Cache cache[64];  // per host thread, device and kernel instantiation
  Cache& cc = cache[g->device < 64 ? g->device : 63];
  if (cc.smem != smem || cc.warps != warps) {
    GS_CUDA_TRY(cudaFuncSetAttribute(k_ingest<CG, R, SMALL, TEN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nb = 0;
    GS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ingest<CG, R, SMALL, TEN>, warps * 32, smem));
    cc.smem = smem;
    cc.warps = warps;
    cc.blocks = nb > 0 ? nb : 1;
  }
  A.vtenant = TEN ? g->d_vtenant : nullptr;
  A.tenants = TEN ? g->d_ten : nullptr;
  k_ingest<CG, R, SMALL, TEN><<<g->num_sms * cc.blocks, warps * 32, smem, s>>>(A);
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

// shared memory per warp of the packed kernel: the graph's geometry, or the widest need over every
// column count up to the engine's widest tenant
uint32_t packed_warp_words(const gs_graph* g) {
  if (!g->d_ten) return pack_warp_words(g->geom.num_columns);
  uint32_t w = 0;
  for (uint32_t c = 1; c <= g->ten_max_cols && c <= 32u; c++) w = std::max(w, pack_warp_words(c));
  return w;
}

template <bool TEN>
gs_status launch_ingest_packed(gs_graph* g, uint32_t nv, cudaStream_t s) {
  IngestArgs A;
  A.off = g->d_off; A.choff = g->d_choff; A.nbr = g->d_nbr; A.sk = g->d_sk; A.colmix = g->d_colmix;
  A.status = g->d_status; A.nv = nv; A.V = g->V; A.C = g->geom.num_columns;
  A.bkt = g->geom.bkt_per_col; A.nb = g->geom.num_buckets; A.chunk = g->tune.chunk;
  A.vtenant = TEN ? g->d_vtenant : nullptr;
  A.tenants = TEN ? g->d_ten : nullptr;
  A.warp_words = packed_warp_words(g);
  A.next_chunk = g->d_status + 14;
  A.owner = g->d_owner;
  A.owner_cap = (uint32_t)g->owner_cap;
  const int warps = std::min(kPackMaxThreads / 32, (int)g->tune.warps_per_block);
  const size_t smem = (size_t)warps * A.warp_words * sizeof(uint4);
  struct Cache { size_t smem = 0; int warps = 0; int blocks = 0; };
  static thread_local Cache cache[64];  // per host thread, device and kernel instantiation
  Cache& cc = cache[g->device < 64 ? g->device : 63];
  if (cc.smem != smem || cc.warps != warps) {
    GS_CUDA_TRY(cudaFuncSetAttribute(k_ingest_packed<TEN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nb = 0;
    GS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ingest_packed<TEN>, warps * 32, smem));
    cc.smem = smem;
    cc.warps = warps;
    cc.blocks = nb > 0 ? nb : 1;
  }
  k_ingest_packed<TEN><<<g->num_sms * cc.blocks, warps * 32, smem, s>>>(A);
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

template <int CG, bool SMALL, bool TEN>
gs_status launch_ingest_r(gs_graph* g, uint32_t nv, cudaStream_t s) {
  switch (g->tune.reg_depth) {
    case 0:
      if constexpr (CG == 1) return launch_ingest_packed<TEN>(g, nv, s);
      else return launch_ingest<CG, 0, SMALL, TEN>(g, nv, s);
    case 1: return launch_ingest<CG, 1, SMALL, TEN>(g, nv, s);
    case 3: return launch_ingest<CG, 3, SMALL, TEN>(g, nv, s);
    default: return launch_ingest<CG, 2, SMALL, TEN>(g, nv, s);
  }
}

template <int CG, bool TEN>
gs_status launch_ingest_s(gs_graph* g, uint32_t nv, bool small, cudaStream_t s) {
  return small ? launch_ingest_r<CG, true, TEN>(g, nv, s) : launch_ingest_r<CG, false, TEN>(g, nv, s);
}

template <bool COMPACT>
gs_status launch_part_scatter_staged(const uint2* p, uint64_t m, const PairTag& t, uint32_t lb, uint32_t H,
                                     uint32_t* bkt, uint2* part, uint64_t cap, uint32_t* status,
                                     const uint32_t* blockhist, cudaStream_t s) {
  const size_t smem = part_scatter_staged_smem(H);
  static thread_local size_t smem_set[64] = {};
  int dev = 0;
  GS_CUDA_TRY(cudaGetDevice(&dev));
  if (smem_set[dev & 63] < smem) {
    GS_CUDA_TRY(cudaFuncSetAttribute(k_part_scatter_staged<COMPACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    smem_set[dev & 63] = smem;
  }
  const unsigned tiles = (unsigned)((m + kPartEdges - 1) / kPartEdges);
  k_part_scatter_staged<COMPACT><<<tiles, kPartThreads, smem, s>>>(p, m, t, lb, H, bkt, part, cap, status, blockhist);
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

gs_status launch_vert_scatter_sorted(const uint2* part, const uint32_t* bkt, uint32_t H, uint32_t lb, uint32_t* cursor,
                                     uint32_t* nbr, uint64_t cap, uint32_t* status, const uint32_t* chunkhist, int grid,
                                     cudaStream_t s) {
  const size_t smem = vert_scatter_sorted_smem(lb);
  static thread_local size_t smem_set[64] = {};
  int dev = 0;
  GS_CUDA_TRY(cudaGetDevice(&dev));
  if (smem_set[dev & 63] < smem) {
    GS_CUDA_TRY(cudaFuncSetAttribute(k_vert_scatter_sorted, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    smem_set[dev & 63] = smem;
  }
  k_vert_scatter_sorted<<<grid, kPartThreads, smem, s>>>(reinterpret_cast<const uint32_t*>(part), bkt, H, lb, cursor,
                                                          nbr, cap, status, chunkhist);
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

// records partitioned by key bucket (pass 1 output) and the bucket tables
static gs_status ensure_partition_scratch(gs_graph* g, uint64_t records) {
  const uint64_t nv = (uint64_t)g->num_levels * g->V;
  if (!g->d_bkt) {
    uint32_t lb = 9;
    while ((nv >> lb) >= (uint64_t)kMaxBuckets) lb++;
    g->part_lb = lb;
    g->part_buckets = (uint32_t)((nv + (1ull << lb) - 1) >> lb);
    GS_CUDA_TRY(cudaMalloc(&g->d_bkt, (4 * (size_t)g->part_buckets + 2) * sizeof(uint32_t)));
  }
  if (g->part_cap < records) {
    cudaFree(g->d_part);
    g->d_part = nullptr;
    g->part_cap = 0;
    GS_CUDA_TRY(cudaMalloc(&g->d_part, records * sizeof(uint2)));
    g->part_cap = records;
  }
  return GS_OK;
}

// per-block bucket counts for a pass of m edges (untagged passes; null when the table would be too big)
static gs_status ensure_blockhist(gs_graph* g, uint64_t m, uint32_t** out) {
  *out = nullptr;
  const uint64_t words = (m + kPartEdges - 1) / kPartEdges * (uint64_t)g->part_buckets;
  if (words == 0 || words > kMaxBlockHistWords) return GS_OK;
  if (g->blockhist_cap < words) {
    cudaFree(g->d_blockhist);
    g->d_blockhist = nullptr;
    g->blockhist_cap = 0;
    GS_CUDA_TRY(cudaMalloc(&g->d_blockhist, (size_t)words * sizeof(uint32_t)));
    g->blockhist_cap = words;
  }
  *out = g->d_blockhist;
  return GS_OK;
}

// per-chunk vertex counts of pass 2 for `records` one-word records (null when the table would be too big)
static gs_status ensure_chunkhist(gs_graph* g, uint64_t records, uint32_t** out) {
  *out = nullptr;
  // chunks: every bucket's records cut into kVertChunk pieces, at most one partial piece per bucket
  const uint64_t chunks = records / kVertChunk + g->part_buckets + 1;
  const uint64_t words = chunks << g->part_lb;
  if (records == 0 || words > kMaxChunkHistWords) return GS_OK;
  if (g->chunkhist_cap < words) {
    cudaFree(g->d_chunkhist);
    g->d_chunkhist = nullptr;
    g->chunkhist_cap = 0;
    GS_CUDA_TRY(cudaMalloc(&g->d_chunkhist, (size_t)words * sizeof(uint32_t)));
    g->chunkhist_cap = words;
  }
  *out = g->d_chunkhist;
  return GS_OK;
}

// The chunk-owner table: a chunk per vertex with records plus one per `chunk` records, the records
// bounded by the neighbour scratch.  A smaller table is never wrong (the sketch update finds the
// chunks past its end by search), so it is not grown while a stream is being captured.
static gs_status ensure_owner_table(gs_graph* g) {
  const uint64_t nv = (uint64_t)g->num_levels * g->V;
  const uint64_t want = std::min<uint64_t>(nv + g->nbr_cap / std::max(1u, g->tune.chunk) + 1, 0xffffffffull);
  if (g->owner_cap >= want || g->capturing) return GS_OK;
  cudaFree(g->d_owner);
  g->d_owner = nullptr;
  g->owner_cap = 0;
  GS_CUDA_TRY(cudaMalloc(&g->d_owner, want * sizeof(uint32_t)));
  g->owner_cap = want;
  return GS_OK;
}

gs_status gs_reserve_ingest(gs_graph* g, uint64_t edges) {
  const uint64_t m = std::min<uint64_t>(edges, g->max_batch_edges);
  GS_TRY(gs_ensure_ingest_scratch(g, std::max<uint64_t>(2 * m, 1)));
  GS_TRY(ensure_partition_scratch(g, std::max<uint64_t>(2 * m, 1)));
  uint32_t* unused = nullptr;
  GS_TRY(ensure_blockhist(g, m, &unused));
  GS_TRY(ensure_chunkhist(g, 2 * m, &unused));
  return ensure_owner_table(g);
}

static gs_status scan_counts(gs_graph* g, uint32_t nv, cudaStream_t s) {
  const uint32_t tiles = (nv + kScanTile - 1) / kScanTile;
  GS_TRY(ensure_owner_table(g));
  k_scan_tiles<<<tiles, kScanThreads, 0, s>>>(g->d_cnt, nv, g->tune.chunk, g->d_off, g->d_choff, g->d_tile);
  k_scan_top<<<1, kScanThreads, 0, s>>>(g->d_tile, tiles, g->d_off, g->d_choff, nv, g->d_status);
  k_scan_add<<<tiles, kScanThreads, 0, s>>>(g->d_off, g->d_choff, g->d_cnt, g->d_tile, nv, g->tune.chunk, g->d_owner,
                                            (uint32_t)g->owner_cap);
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

static gs_status ingest_chunks(gs_graph* g, uint32_t nv, cudaStream_t s) {
  const bool ten = g->d_ten != nullptr;
  const uint32_t cols = ten ? g->ten_max_cols : g->geom.num_columns;
  const bool small = (ten ? g->ten_min_bkt : g->geom.bkt_per_col) < (uint32_t)kSlabDepth;
  if (cols <= 32) return ten ? launch_ingest_s<1, true>(g, nv, small, s) : launch_ingest_s<1, false>(g, nv, small, s);
  if (cols <= 64) return ten ? launch_ingest_s<2, true>(g, nv, small, s) : launch_ingest_s<2, false>(g, nv, small, s);
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
  // records tag into the sketched levels 0..store_first-1 (every level unless the exact tier is adaptive)
  const uint32_t sketched = g->store_first;
  PairTag t;
  t.V = g->V; t.num_levels = sketched; t.L = g->num_subgraphs; t.fixed_level = fixed_level;
  t.cs_mix = gs_seed_mix(g->seed);
  const bool tagged = sketched > 1 && fixed_level < 0;
  const bool no_sketch = fixed_level < 0 && sketched == 0;  // every edge is kept exactly
  for (uint64_t done = 0; done < n;) {
    const uint64_t m = std::min<uint64_t>(n - done, g->max_batch_edges);
    const uint2* p = reinterpret_cast<const uint2*>(d_pairs) + done;
    if (no_sketch) {
      GS_TRY(gs_store_ingest(g, reinterpret_cast<const uint32_t*>(p), m, s));
      GS_TRY(gs_store_maintain(g, s));
      g->records_total += m;
      done += m;
      continue;
    }
    const uint64_t bound = tagged ? std::max<uint64_t>(g->part_cap, 4 * m) : 2 * m;
    GS_TRY(gs_ensure_ingest_scratch(g, tagged ? std::max<uint64_t>(g->nbr_cap, 4 * m) : 2 * m));
    GS_TRY(ensure_partition_scratch(g, bound));
    const uint32_t H = g->part_buckets, lb = g->part_lb;
    const unsigned tiles = (unsigned)((m + kPartEdges - 1) / kPartEdges);
    const int grid2 = g->num_sms * 4;
    // per-block bucket counts handed from the count pass to the staged placement (untagged passes,
    // while the table stays small: tiles x H words)
    uint32_t* blockhist = nullptr;
    if (!tagged) GS_TRY(ensure_blockhist(g, m, &blockhist));
    {
      GsProfScope ps(g, GS_PROF_BUCKET, s, 2);
      GS_CUDA_TRY(cudaMemsetAsync(g->d_bkt, 0, (size_t)H * sizeof(uint32_t), s));
      GS_CUDA_TRY(cudaMemsetAsync(g->d_cnt, 0, (size_t)(nv + 1) * sizeof(uint32_t), s));
      k_part_count<<<tiles, kPartThreads, H * sizeof(uint32_t), s>>>(p, m, t, lb, H, g->d_bkt, g->d_status,
                                                                     tagged ? nullptr : blockhist);
      k_part_scan<<<1, kScanThreads, 0, s>>>(g->d_bkt, H, g->d_status);
      GS_CUDA_TRY(cudaGetLastError());
    }
    if (tagged) {
      // the record count depends on the tags: read it back and grow the scratch if needed
      GS_CUDA_TRY(cudaMemcpyAsync(g->h_status, g->d_status, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      GS_CUDA_TRY(cudaStreamSynchronize(s));
      const uint64_t recs = g->h_status[1];
      if (recs > g->part_cap) GS_TRY(ensure_partition_scratch(g, recs + recs / 8));
      if (recs > g->nbr_cap) GS_TRY(gs_ensure_ingest_scratch(g, recs + recs / 8));
    }
    {
      GsProfScope ps(g, GS_PROF_BUCKET, s, 6);
      // one-word records when a bucket-local key and a neighbour id fit together
      const bool compact = !tagged && (uint64_t)g->V <= (1ull << (32u - lb));
      if (tagged) {
        k_part_scatter<<<tiles, kPartThreads, 2 * H * sizeof(uint32_t), s>>>(p, m, t, lb, H, g->d_bkt, g->d_part,
                                                                             g->part_cap, g->d_status);
      } else if (compact) {
        GS_TRY(launch_part_scatter_staged<true>(p, m, t, lb, H, g->d_bkt, g->d_part, g->part_cap, g->d_status,
                                                blockhist, s));
      } else {
        GS_TRY(launch_part_scatter_staged<false>(p, m, t, lb, H, g->d_bkt, g->d_part, g->part_cap, g->d_status,
                                                 blockhist, s));
      }
      const size_t vc_smem = (1u << lb) * sizeof(uint32_t), vs_smem = 2 * (1u << lb) * sizeof(uint32_t);
      if (compact) {
        uint32_t* chunkhist = nullptr;
        GS_TRY(ensure_chunkhist(g, 2 * m, &chunkhist));
        k_vert_count<true><<<grid2, kPartThreads, vc_smem, s>>>(g->d_part, g->d_bkt, H, lb, g->d_cnt, g->d_status,
                                                               chunkhist);
        GS_TRY(scan_counts(g, nv, s));
        GS_TRY(launch_vert_scatter_sorted(g->d_part, g->d_bkt, H, lb, g->d_cnt, g->d_nbr, g->nbr_cap, g->d_status,
                                          chunkhist, g->num_sms * 3, s));
      } else {
        k_vert_count<false><<<grid2, kPartThreads, vc_smem, s>>>(g->d_part, g->d_bkt, H, lb, g->d_cnt, g->d_status,
                                                                nullptr);
        GS_TRY(scan_counts(g, nv, s));
        k_vert_scatter<false><<<grid2, kPartThreads, vs_smem, s>>>(g->d_part, g->d_bkt, H, lb, g->d_cnt, g->d_nbr,
                                                                   g->nbr_cap, g->d_status);
      }
      GS_CUDA_TRY(cudaGetLastError());
    }
    {
      GsProfScope ps(g, GS_PROF_INGEST, s, 1);
      GS_TRY(ingest_chunks(g, nv, s));
    }
    if (fixed_level < 0) {
      GS_TRY(gs_eager_ingest(g, reinterpret_cast<const uint32_t*>(p), m, s));
      GS_TRY(gs_store_ingest(g, reinterpret_cast<const uint32_t*>(p), m, s));
      GS_TRY(gs_store_maintain(g, s));
    }
    g->records_total += m;
    done += m;
  }
  return GS_OK;
}

gs_status gs_ingest_device_batches(gs_graph* g, uint32_t level, const uint32_t* d_srcs,
                                   const uint64_t* d_starts, const uint64_t* d_sizes, uint32_t nbat,
                                   const uint32_t* d_dsts, cudaStream_t s, uint64_t max_records) {
  if (nbat == 0) return GS_OK;
  // directed one-sided updates: the eager DSU cannot follow them
  GS_TRY(gs_eager_invalidate(g, s));
  const uint32_t nv = g->num_levels * g->V;
  GS_TRY(gs_ensure_ingest_scratch(g, std::max<uint64_t>(max_records, 1)));
  GS_CUDA_TRY(cudaMemsetAsync(g->d_cnt, 0, (size_t)(nv + 1) * sizeof(uint32_t), s));
  {
    GsProfScope ps(g, GS_PROF_BUCKET, s, 4);
    k_count_batches<<<grid_for(g, nbat, 256), 256, 0, s>>>(d_srcs, d_sizes, nbat, g->V, level, g->d_cnt, g->d_status);
    GS_CUDA_TRY(cudaGetLastError());
    GS_TRY(scan_counts(g, nv, s));
  }
  // the record count sizes the neighbour scratch: a caller that knows a bound (the host path: the
  // sum of the batch sizes) spares the read-back and its wait
  uint64_t recs = max_records;
  if (!max_records) {
    GS_CUDA_TRY(cudaMemcpyAsync(g->h_status, g->d_status, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GS_CUDA_TRY(cudaStreamSynchronize(s));
    recs = g->h_status[1];
    if (recs > g->nbr_cap) GS_TRY(gs_ensure_ingest_scratch(g, recs));
  }
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

// ---- ingest over caller-supplied scratch ----

size_t gs_scratch_ingest_smem_bytes(const GsGeom& geom, uint32_t warps) {
  return ingest_smem_bytes(geom.num_columns <= 32 ? 1 : 2, 1, (int)warps);
}

namespace {

template <int CG, bool SMALL>
gs_status launch_ingest_scratch(const GsScratchIngest& x, cudaStream_t s) {
  IngestArgs A;
  A.off = x.off; A.choff = x.choff; A.nbr = x.nbr; A.sk = x.sketches; A.colmix = x.colmix;
  A.status = x.status; A.nv = x.geom.V; A.V = x.geom.V; A.C = x.geom.num_columns;
  A.bkt = x.geom.bkt_per_col; A.nb = x.geom.num_buckets; A.chunk = x.chunk;
  A.vtenant = nullptr;
  A.tenants = nullptr;
  A.warp_words = 0;
  A.next_chunk = nullptr;
  A.owner = nullptr;
  A.owner_cap = 0;
  const size_t smem = ingest_smem_bytes(CG, 1, (int)x.warps);
  int nb = 0;
  GS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ingest<CG, 1, SMALL, false>, (int)x.warps * 32, smem));
  k_ingest<CG, 1, SMALL, false><<<x.num_sms * (nb > 0 ? nb : 1), x.warps * 32, smem, s>>>(A);
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

}  // namespace

gs_status gs_ingest_pairs_on_scratch(const GsScratchIngest& x, cudaStream_t s) {
  if (x.n == 0) return GS_OK;
  const uint32_t nv = x.geom.V;
  PairTag t;
  t.V = nv; t.num_levels = 1; t.L = 1; t.fixed_level = -1; t.cs_mix = 0;
  const uint32_t H = x.part_buckets, lb = x.part_lb;
  const unsigned tiles = (unsigned)((x.n + kPartEdges - 1) / kPartEdges);
  const int grid2 = x.num_sms * 4;
  // everything that must start at zero: error word and totals, bucket totals, vertex counts
  GS_CUDA_TRY(cudaMemsetAsync(x.status, 0, 16 * sizeof(uint32_t), s));
  GS_CUDA_TRY(cudaMemsetAsync(x.bkt, 0, (size_t)H * sizeof(uint32_t), s));
  GS_CUDA_TRY(cudaMemsetAsync(x.cnt, 0, (size_t)(nv + 1) * sizeof(uint32_t), s));
  const uint2* p = reinterpret_cast<const uint2*>(x.pairs);
  k_part_count<<<tiles, kPartThreads, H * sizeof(uint32_t), s>>>(p, x.n, t, lb, H, x.bkt, x.status, nullptr);
  k_part_scan<<<1, kScanThreads, 0, s>>>(x.bkt, H, x.status);
  k_part_scatter<<<tiles, kPartThreads, 2 * H * sizeof(uint32_t), s>>>(p, x.n, t, lb, H, x.bkt, x.part,
                                                                       x.records_cap, x.status);
  k_vert_count<false><<<grid2, kPartThreads, (1u << lb) * sizeof(uint32_t), s>>>(x.part, x.bkt, H, lb, x.cnt, x.status,
                                                                                nullptr);
  const uint32_t stiles = (nv + kScanTile - 1) / kScanTile;
  k_scan_tiles<<<stiles, kScanThreads, 0, s>>>(x.cnt, nv, x.chunk, x.off, x.choff, x.tile);
  k_scan_top<<<1, kScanThreads, 0, s>>>(x.tile, stiles, x.off, x.choff, nv, x.status);
  k_scan_add<<<stiles, kScanThreads, 0, s>>>(x.off, x.choff, x.cnt, x.tile, nv, x.chunk, nullptr, 0u);
  k_vert_scatter<false><<<grid2, kPartThreads, 2 * (1u << lb) * sizeof(uint32_t), s>>>(x.part, x.bkt, H, lb, x.cnt, x.nbr,
                                                                                x.records_cap, x.status);
  GS_CUDA_TRY(cudaGetLastError());
  const bool small = x.geom.bkt_per_col < (uint32_t)kSlabDepth;
  if (x.geom.num_columns <= 32)
    return small ? launch_ingest_scratch<1, true>(x, s) : launch_ingest_scratch<1, false>(x, s);
  return small ? launch_ingest_scratch<2, true>(x, s) : launch_ingest_scratch<2, false>(x, s);
}
