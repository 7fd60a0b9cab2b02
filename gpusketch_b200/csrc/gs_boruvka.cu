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
// All rounds run inside one persistent kernel (k_boruvka), so a query is one launch and one
// read-back instead of a host round trip per round.  Its blocks are co-resident (cooperative
// launch) and meet at a grid barrier between phases; every barrier wait is bounded and reports
// GS_DEV_ERR_TIMEOUT instead of spinning forever.  Several independent graphs ("tenants", each with
// its own geometry and seed) can share one launch: their vertices are disjoint ranges of one vertex
// space, their rounds advance together, and a tenant whose round was unmodified stops taking part,
// so each tenant's partition, round count and out-of-samples status equal a query run alone.
//
// Per round (five grid barriers):
//   sizes       component sizes from the compressed parent array (warp-aggregated atomics); the
//               size array also freezes the round's root set for sampling and unions
//   accumulate  warps take runs of vertices from a shared counter, stage the members' column r and
//               deterministic bucket in shared memory with cp.async, and XOR them into a register
//               accumulator per component, flushed with red.global.xor when the component changes
//   sample      round 0: every vertex samples its own sketch (an octet of lanes per vertex for one
//               graph, a thread per vertex for many); later rounds: one warp per listed root, lane j
//               checking bucket j (and j+32) with one XXH3 each (Bucket_Boruvka::is_good,
//               include/bucket.h:65-67).  The deterministic bucket is zero / good first, else the first
//               good bucket by depth (Sketch::sample, src/sketch.cpp:110-132); the component's
//               accumulator row is zeroed once read, so rows are all zero between rounds and launches
//   union       one thread per root unions its sampled edge, so thousands of DSU walks overlap
//   compress    full path compression, sizes cleared, per-tenant stop / out-of-samples decisions
// DSU: CAS hooking of the larger root under the smaller (include/dsu.h:155-167 unions by random
// priority instead), so every component's root is its minimum vertex id and labels are deterministic;
// every walk is bounded by V+64 steps and reports GS_DEV_ERR_DSU_LIMIT.
#include "gs_dsu.cuh"
#include "gs_internal.h"

namespace {

constexpr uint32_t kGood = 0, kZero = 1, kFail = 2;
constexpr uint32_t kAccRun = 16;                 // vertices a warp stages in shared memory at once
constexpr uint32_t kAccGrab = 64;                // vertices a warp takes from the shared work counter
constexpr uint32_t kThreads = 256;
constexpr uint32_t kWarps = kThreads / 32;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }


// loads of data written by other blocks earlier in the same launch bypass L1
__device__ __forceinline__ GsBucket ld_bucket_cg(const GsBucket* p) {
  const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(p));
  return GsBucket{v.x, v.y};
}

// 16-byte global -> shared copy that completes asynchronously (waited for with cp_async_wait_all)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ bool is_good(const GsBucket& b, uint64_t csmix) {
  return gs_hash_tail(gs_key_mix(b.alpha) ^ csmix) == b.gamma;
}

// Sketch::sample on one column: all lanes of the warp call it and get the same answer.  The
// deterministic bucket and the first 32 column buckets are loaded together.
__device__ __forceinline__ void sample_warp(const GsBucket* col, const GsBucket* det, uint32_t bkt, uint64_t csmix,
                                            uint32_t* code, uint64_t* idx) {
  const uint32_t lane = lane_id();
  const GsBucket d = ld_bucket_cg(det);
  GsBucket b = GsBucket{0, 0};
  if (lane < bkt) b = ld_bucket_cg(col + lane);
  if (d.alpha == 0 && d.gamma == 0) { *code = kZero; *idx = 0; return; }
  if (is_good(d, csmix)) { *code = kGood; *idx = d.alpha; return; }
  for (uint32_t j0 = 0; j0 < bkt; j0 += 32) {
    const uint32_t j = j0 + lane;
    if (j0 > 0 && j < bkt) b = ld_bucket_cg(col + j);
    const bool good = j < bkt && is_good(b, csmix);
    const uint32_t m = __ballot_sync(0xffffffffu, good);
    if (m) {
      *code = kGood;
      *idx = __shfl_sync(0xffffffffu, b.alpha, __ffs(m) - 1);
      return;
    }
  }
  *code = kFail;
  *idx = 0;
}

// Sketch::sample by one thread (round 0 of multi-graph launches, whose vertices are mostly sparse
// and decide at the deterministic bucket): the column by depth, four buckets per batch of loads.
__device__ __forceinline__ void sample_thread(const GsBucket* col, const GsBucket* det, uint32_t bkt, uint64_t csmix,
                                              uint32_t* code, uint64_t* idx) {
  const GsBucket d = ld_bucket_cg(det);
  if (d.alpha == 0 && d.gamma == 0) { *code = kZero; *idx = 0; return; }
  if (is_good(d, csmix)) { *code = kGood; *idx = d.alpha; return; }
  for (uint32_t j0 = 0; j0 < bkt; j0 += 4) {
    GsBucket b[4];
#pragma unroll
    for (int k = 0; k < 4; k++) b[k] = j0 + k < bkt ? ld_bucket_cg(col + j0 + k) : GsBucket{0, 0};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if (j0 + k < bkt && is_good(b[k], csmix)) {
        *code = kGood;
        *idx = b[k].alpha;
        return;
      }
    }
  }
  *code = kFail;
  *idx = 0;
}

// Sketch::sample by an octet of lanes (round 0, where every vertex samples its own sketch: four
// vertices per warp).  Lane k of the octet checks depths k, k+8, ...; an octet's answer is the lowest
// good depth among its lanes.  The octets of a warp may belong to graphs with different bkt, so the
// pass count is the warp's largest bkt: every lane runs the same passes and reaches every
// full-warp collective.
__device__ __forceinline__ void sample_octet(const GsBucket* col, const GsBucket* det, uint32_t bkt, uint64_t csmix,
                                             bool active, uint32_t* code, uint64_t* idx) {
  const uint32_t lane = lane_id(), sub = lane & 7u, oct = lane >> 3;
  bool decided = !active;
  *code = kFail;
  *idx = 0;
  if (active) {
    const GsBucket d = ld_bucket_cg(det);
    if (d.alpha == 0 && d.gamma == 0) { *code = kZero; decided = true; }
    else if (is_good(d, csmix)) { *code = kGood; *idx = d.alpha; decided = true; }
  }
  const uint32_t bmax = __reduce_max_sync(0xffffffffu, bkt);
  for (uint32_t j0 = 0; j0 < bmax; j0 += 8) {
    if (__all_sync(0xffffffffu, decided)) break;
    const uint32_t j = j0 + sub;
    GsBucket b = GsBucket{0, 0};
    const bool look = !decided && j < bkt;
    if (look) b = ld_bucket_cg(col + j);
    const uint32_t m = __ballot_sync(0xffffffffu, look && is_good(b, csmix));
    const uint32_t mine = (m >> (8u * oct)) & 0xffu;
    const uint64_t a = __shfl_sync(0xffffffffu, b.alpha, mine ? 8u * oct + (uint32_t)(__ffs(mine) - 1) : lane);
    if (!decided && mine) {
      *code = kGood;
      *idx = a;
      decided = true;
    }
  }
}

// Grid-wide barrier of a co-resident launch.  Returns false when any block gave up waiting.  The
// waiting thread backs off exponentially (32 ns .. 1 us) so that hundreds of pollers do not saturate
// the L2 slice that holds the generation word.
// wait_ns: how long (summed sleep time) a block waits for the others before it reports
// GS_DEV_ERR_TIMEOUT and gives up
__device__ bool grid_sync(uint32_t* count, uint32_t* gen, uint32_t* err, uint64_t wait_ns) {
  __shared__ uint32_t s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ok = 1;
    const uint32_t g = ld_volatile(gen);
    __threadfence();
    if (atomicAdd(count, 1u) == gridDim.x - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      uint32_t sleep_ns = 32, it = 0;
      uint64_t waited = 0;
      while (ld_volatile(gen) == g) {
        __nanosleep(sleep_ns);
        waited += sleep_ns;
        // back-off capped at 256 ns: a block that waited long notices the release within a
        // quarter microsecond (1024 ns made the 10-round query 1% slower)
        if (sleep_ns < 256) sleep_ns <<= 1;
        if ((++it & 63u) == 0 && (ld_volatile(err) & GS_DEV_ERR_TIMEOUT)) { ok = 0; break; }
        if (waited > wait_ns) {
          atomicOr(err, (uint32_t)GS_DEV_ERR_TIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    s_ok = ok && !(ld_volatile(err) & GS_DEV_ERR_TIMEOUT);
  }
  __syncthreads();
  return s_ok != 0;
}

struct BorArgs {
  const GsBucket* sk;          // sketch base the tenants' sk_off index into
  const GsBorTenant* tenants;  // [T] (device), or nullptr: the single tenant t0
  GsBorTenant t0;
  const uint32_t* vtenant;     // [V] tenant of each vertex, nullptr when T == 1
  uint32_t T, V, W;            // W: accumulator row width, max bkt_per_col + 1
  uint32_t vlo;                // the kernel works on vertices [vlo, V)
  uint32_t max_rounds;         // max num_samples over the tenants
  uint32_t* parent;            // [V]
  uint32_t* size;              // [V]
  GsBucket* acc;               // [V][W]
  uint64_t* samp;              // [V] sampled edge of each root this round (global ids), ~0 = none
  uint32_t* roots;             // [V] this round's roots, status[3] of them
  uint32_t* forest;            // [2 * forest_cap]
  uint32_t forest_cap;
  uint32_t* status;            // [0] error bits [3] roots [4] forest edges [5] active tenants [6,7] barrier
                               // [12] accumulate work counter
  uint32_t* tstate;            // [T][4]: done, modified this round, rounds, out of samples
  uint64_t wait_ns;            // grid-barrier wait limit
  uint32_t complement;         // every tenant's sketch set XORs to zero: see the accumulate phase
  unsigned long long* largest; // [T] (size << 32) | ~root of each tenant's largest component this round
};

// root of tenant t's largest component this round, or ~0 when it has no component of two or more
__device__ __forceinline__ uint32_t largest_root(const BorArgs& A, uint32_t t) {
  const unsigned long long k = *reinterpret_cast<const volatile unsigned long long*>(A.largest + t);
  return (k >> 32) > 1ull ? 0xffffffffu - (uint32_t)k : 0xffffffffu;
}

__device__ __forceinline__ const GsBorTenant& tenant_of(const BorArgs& A, uint32_t t) {
  return A.tenants ? A.tenants[t] : A.t0;
}

__device__ __forceinline__ void flush_acc(const BorArgs& A, uint32_t cur, uint32_t w, const uint64_t* a,
                                          const uint64_t* gm) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint32_t j = lane_id() + 32u * k;
    if (j < w && (a[k] | gm[k])) {
      atomicXor(reinterpret_cast<unsigned long long*>(&A.acc[(size_t)cur * A.W + j].alpha), (unsigned long long)a[k]);
      atomicXor(reinterpret_cast<unsigned long long*>(&A.acc[(size_t)cur * A.W + j].gamma), (unsigned long long)gm[k]);
    }
  }
}

// The accumulators a warp still holds at the end of the accumulate phase, flushed once per block:
// warps of a block that hold the same component's row (every warp holds the largest component's)
// combine them in shared memory, so one warp per block and component issues the global XORs instead
// of every warp - the atomics on that row serialize in L2.  Called by every thread of the block.
__device__ void block_flush(const BorArgs& A, uint32_t root, uint32_t w, const uint64_t* a, const uint64_t* gm,
                            uint32_t* s_root, GsBucket* stage0) {
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
  GsBucket* row = stage0 + (size_t)wib * kAccRun * A.W;
  if (lane == 0) s_root[wib] = root;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint32_t j = lane + 32u * k;
    if (j < w) row[j] = GsBucket{a[k], gm[k]};
  }
  __syncthreads();
  if (root != 0xffffffffu) {
    bool leader = true;
    for (uint32_t o = 0; o < wib; o++) leader = leader && s_root[o] != root;
    if (leader) {
      uint64_t x[3] = {a[0], a[1], a[2]}, y[3] = {gm[0], gm[1], gm[2]};
      for (uint32_t o = wib + 1; o < nw; o++) {
        if (s_root[o] != root) continue;
        const GsBucket* other = stage0 + (size_t)o * kAccRun * A.W;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const uint32_t j = lane + 32u * k;
          if (j < w) { x[k] ^= other[j].alpha; y[k] ^= other[j].gamma; }
        }
      }
      flush_acc(A, root, w, x, y);
    }
  }
  __syncthreads();
}

// done flags of the tenants, copied from tstate into shared memory once per round
__device__ __forceinline__ void snapshot_done(const BorArgs& A, uint32_t* s_done) {
  for (uint32_t t = threadIdx.x; t < A.T; t += blockDim.x) s_done[t] = ld_volatile(&A.tstate[4 * t]);
  __syncthreads();
}

// Dynamic shared memory: the tenants' done flags (T words, padded to 16 bytes), then one staging
// area of kAccRun x W buckets per warp.
// three blocks per SM, as shared memory allows: the bound keeps the registers at 78 (122 without it,
// which left two blocks per SM), with no spills
__global__ void __launch_bounds__(kThreads, 3) k_boruvka(const BorArgs A) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ uint32_t s_root[kWarps];
  uint32_t* s_done = smem;
  GsBucket* stage = reinterpret_cast<GsBucket*>(smem + ((A.T + 3u) & ~3u)) + (threadIdx.x >> 5) * kAccRun * A.W;
  uint32_t* err = A.status;
  uint32_t* nroots_p = A.status + 3;
  uint32_t* acc_next = A.status + 12;  // accumulate work counter, zero at launch and after every round
  uint32_t* bcount = A.status + 6;
  uint32_t* bgen = A.status + 7;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gthreads = gridDim.x * blockDim.x;
  const uint32_t gwarp = gtid >> 5, gwarps = gthreads >> 5, lane = lane_id();
  const uint32_t limit = A.V + 64;
  const uint32_t span = A.V - A.vlo;

  for (uint32_t v = A.vlo + gtid; v < A.V; v += gthreads) A.parent[v] = v;
  if (gtid == 0) *nroots_p = 0;
  if (A.complement)
    for (uint32_t t = gtid; t < A.T; t += gthreads) A.largest[t] = 0ull;
  if (!grid_sync(bcount, bgen, err, A.wait_ns)) return;

  for (uint32_t round = 0; round < A.max_rounds; round++) {
    snapshot_done(A, s_done);
    if (round > 0) {
      // ---- sizes of the round's components (size[] was zeroed by the previous compress); the
      //      first adder of each root appends it to the root list ----
      for (uint32_t base = A.vlo + blockIdx.x * blockDim.x; base < A.V; base += gthreads) {
        const uint32_t v = base + threadIdx.x;
        uint32_t r = 0xffffffffu;
        if (v < A.V) {
          const uint32_t t = A.vtenant ? A.vtenant[v] : 0u;
          if (!s_done[t]) r = __ldcg(&A.parent[v]);
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, r);
        bool fresh = false;
        if (r != 0xffffffffu && lane == (uint32_t)(__ffs(peers) - 1))
          fresh = atomicAdd(&A.size[r], (uint32_t)__popc(peers)) == 0u;
        const uint32_t fm = __ballot_sync(0xffffffffu, fresh);
        if (fm) {
          uint32_t at = 0;
          if (lane == (uint32_t)(__ffs(fm) - 1)) at = atomicAdd(nroots_p, (uint32_t)__popc(fm));
          at = __shfl_sync(0xffffffffu, at, __ffs(fm) - 1);
          if (fresh) A.roots[at + __popc(fm & ((1u << lane) - 1u))] = r;
        }
      }
      if (!grid_sync(bcount, bgen, err, A.wait_ns)) return;

      // ---- complement: each tenant's largest component this round (ties to the smallest root) ----
      if (A.complement) {
        const uint32_t nr = ld_volatile(nroots_p);
        if (A.T == 1) {
          unsigned long long best = 0ull;
          for (uint32_t k = gtid; k < nr; k += gthreads) {
            const uint32_t r = __ldcg(&A.roots[k]);
            const unsigned long long key = ((unsigned long long)__ldcg(&A.size[r]) << 32) | (0xffffffffu - r);
            best = key > best ? key : best;
          }
          for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
            best = other > best ? other : best;
          }
          if (lane == 0 && best) atomicMax(A.largest, best);
        } else {
          for (uint32_t k = gtid; k < nr; k += gthreads) {
            const uint32_t r = __ldcg(&A.roots[k]);
            const uint32_t sz = __ldcg(&A.size[r]);
            if (sz > 1u) atomicMax(A.largest + A.vtenant[r], ((unsigned long long)sz << 32) | (0xffffffffu - r));
          }
        }
        if (!grid_sync(bcount, bgen, err, A.wait_ns)) return;
      }

      // ---- accumulate column r + the deterministic bucket per component ----
      // Warps take runs of kAccGrab vertices from a shared counter (finished tenants' vertices cost
      // almost nothing, so fixed slices would leave most warps idle at the barrier) and walk each
      // run kAccRun at a time: the columns of the members are copied into shared memory with
      // cp.async (all in flight together), then folded in vertex order into a register accumulator
      // that is flushed with red.global.xor when the component changes.  A vertex whose root is
      // another vertex is in a component of two or more, so only roots read their own size: no load
      // hammers a giant component's root.
      //
      // Complement (sketch sets that XOR to zero, because every update reached both endpoints): the
      // XOR of ALL of a graph's vertex sketches is zero, so its largest component's merged column
      // equals the XOR of the columns of every vertex of the graph outside it.  The largest
      // component's members are then skipped, and every other vertex - singletons included - is
      // folded into its graph's largest-component row as well as its own.  A round reads the vertices
      // outside the largest components instead of all of them.
      {
        uint32_t cur = 0xffffffffu, w = 0;
        uint64_t a[3] = {0, 0, 0}, gm[3] = {0, 0, 0};
        uint32_t ccur = 0xffffffffu, cw = 0;              // the largest-component row being folded
        uint64_t ca[3] = {0, 0, 0}, cg[3] = {0, 0, 0};
        // One graph with the complement: most vertices cost one parent load, so runs are assigned to
        // warps in a fixed stride (measured 0.39 vs 0.52 ms per V=2^17 query against the counter).
        // Otherwise warps take runs from the shared counter, because finished tenants' vertices cost
        // almost nothing and fixed slices would leave warps idle (the 256-tenant query: 2.35 ms per
        // query with the counter, 2.95 with the stride; reading the counter before the atomic, to keep
        // warps that find the work gone off it, made it 3.05).
        const bool strided = A.complement && A.T == 1;
        uint32_t stride_next = gwarp * kAccRun;
        const uint32_t grab = strided ? kAccRun : kAccGrab;   // vertices per taken piece of work
        for (;;) {
          uint32_t g0 = 0;
          if (strided) {
            g0 = stride_next;
            stride_next += gwarps * kAccRun;
          } else {
            if (lane == 0) g0 = atomicAdd(acc_next, grab);
            g0 = __shfl_sync(0xffffffffu, g0, 0);
          }
          if (g0 >= span) break;
          const uint32_t w1 = A.vlo + min(span, g0 + grab);
        for (uint32_t start = A.vlo + g0; start < w1; start += kAccRun) {
          const uint32_t n = min(kAccRun, w1 - start);
          uint32_t rt = 0xffffffffu, tt = 0, cb = 0xffffffffu;
          bool outside = false;   // folded into its graph's largest-component row cb (complement)
          if (lane < n) {
            const uint32_t v = start + lane;
            tt = A.vtenant ? A.vtenant[v] : 0u;
            if (!s_done[tt]) {
              const uint32_t r = __ldcg(&A.parent[v]);
              if (A.complement) cb = largest_root(A, tt);
              if (cb != 0xffffffffu) {
                outside = r != cb;
                if (outside && (r != v || __ldcg(&A.size[v]) > 1u)) rt = r;
              } else if (r != v || __ldcg(&A.size[v]) > 1u) {
                rt = r;
              }
            }
          }
          const uint32_t own = __ballot_sync(0xffffffffu, rt != 0xffffffffu);
          const uint32_t outm = __ballot_sync(0xffffffffu, outside);
          const uint32_t live = own | outm;
          for (uint32_t m = live; m;) {
            const uint32_t i = __ffs(m) - 1;
            m &= m - 1;
            const GsBorTenant& T = tenant_of(A, __shfl_sync(0xffffffffu, tt, i));
            const GsBucket* vb = A.sk + T.sk_off + (size_t)(start + i - T.vbase) * T.nb;
            for (uint32_t j = lane; j <= T.bkt; j += 32)
              cp_async16(stage + i * A.W + j, j < T.bkt ? vb + (size_t)round * T.bkt + j : vb + (T.nb - 1));
          }
          cp_async_wait_all();
          __syncwarp();
          for (uint32_t m = live; m;) {
            const uint32_t i = __ffs(m) - 1;
            m &= m - 1;
            const uint32_t wi = tenant_of(A, __shfl_sync(0xffffffffu, tt, i)).bkt + 1;
            if ((outm >> i) & 1u) {
              const uint32_t ci = __shfl_sync(0xffffffffu, cb, i);
              if (ci != ccur) {
                if (ccur != 0xffffffffu) flush_acc(A, ccur, cw, ca, cg);
                ccur = ci;
                cw = wi;
#pragma unroll
                for (int k = 0; k < 3; k++) ca[k] = cg[k] = 0;
              }
#pragma unroll
              for (int k = 0; k < 3; k++) {
                const uint32_t j = lane + 32u * k;
                if (j < wi) {
                  const GsBucket b = stage[i * A.W + j];
                  ca[k] ^= b.alpha;
                  cg[k] ^= b.gamma;
                }
              }
            }
            if (!((own >> i) & 1u)) continue;
            const uint32_t root = __shfl_sync(0xffffffffu, rt, i);
            if (root != cur) {
              if (cur != 0xffffffffu) flush_acc(A, cur, w, a, gm);
              cur = root;
              w = wi;
#pragma unroll
              for (int k = 0; k < 3; k++) a[k] = gm[k] = 0;
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {
              const uint32_t j = lane + 32u * k;
              if (j < w) {
                const GsBucket b = stage[i * A.W + j];
                a[k] ^= b.alpha;
                gm[k] ^= b.gamma;
              }
            }
          }
          __syncwarp();
        }
        }
        // the warps' last rows: combined per block (the largest component's row, or with the direct
        // accumulation the giant component's, is held by nearly every warp)
        block_flush(A, cur, w, a, gm, s_root, stage - (threadIdx.x >> 5) * kAccRun * A.W);
        block_flush(A, ccur, cw, ca, cg, s_root, stage - (threadIdx.x >> 5) * kAccRun * A.W);
      }
      if (!grid_sync(bcount, bgen, err, A.wait_ns)) return;
    }

    // ---- sample every root into samp[root]: roots spread over the warps by list position ----
    // The accumulator row of a sampled component is zeroed after reading, so every row is zero
    // again when the round ends (and at the start of the next launch).
    const uint32_t nroots = round == 0 ? span : ld_volatile(nroots_p);
    if (round == 0 && A.T > 1) {
      // every vertex samples its own sketch: one thread each (many sparse graphs)
      for (uint32_t v = A.vlo + gtid; v < A.V; v += gthreads) {
        const uint32_t t = A.vtenant ? A.vtenant[v] : 0u;
        if (s_done[t]) continue;
        const GsBorTenant& T = tenant_of(A, t);
        const uint32_t col = T.round0_col;
        if (col >= T.ns) {  // OutOfSamplesException
          A.tstate[4 * t + 3] = 1u;
          continue;
        }
        const GsBucket* own = A.sk + T.sk_off + (size_t)(v - T.vbase) * T.nb;
        uint32_t code;
        uint64_t idx;
        sample_thread(own + (size_t)col * T.bkt, own + (T.nb - 1), T.bkt, T.csmix, &code, &idx);
        uint64_t e = ~0ull;
        if (code == kFail) {
          A.tstate[4 * t + 1] = 1u;
        } else if (code == kGood) {
          const uint32_t s = (uint32_t)(idx >> 32), d = (uint32_t)idx;
          if (s < T.V && d < T.V && s != d) e = ((uint64_t)(T.vbase + s) << 32) | (T.vbase + d);
        }
        A.samp[v] = e;
      }
    } else if (round == 0) {
      // every vertex samples its own sketch: an octet of lanes each, four vertices per warp (one
      // graph, whose high-degree vertices find their first good bucket deep in the column)
      for (uint32_t base = A.vlo + gwarp * 4u; base < A.V; base += gwarps * 4u) {
        const uint32_t v = base + (lane >> 3);
        bool active = v < A.V;
        uint32_t t = 0;
        if (active) {
          t = A.vtenant ? A.vtenant[v] : 0u;
          active = !s_done[t];
        }
        const GsBorTenant& T = tenant_of(A, active ? t : 0u);
        const uint32_t col = T.round0_col;
        const bool oos = active && col >= T.ns;  // OutOfSamplesException
        if (oos && (lane & 7u) == 0) A.tstate[4 * t + 3] = 1u;
        const GsBucket* own = A.sk + T.sk_off + (size_t)((active ? v : T.vbase) - T.vbase) * T.nb;
        uint32_t code;
        uint64_t idx;
        sample_octet(own + (size_t)(oos ? 0u : col) * T.bkt, own + (T.nb - 1), T.bkt, T.csmix, active && !oos, &code,
                     &idx);
        if (active && !oos && (lane & 7u) == 0) {
          uint64_t e = ~0ull;
          if (code == kFail) {
            A.tstate[4 * t + 1] = 1u;
          } else if (code == kGood) {
            const uint32_t s = (uint32_t)(idx >> 32), d = (uint32_t)idx;
            if (s < T.V && d < T.V && s != d) e = ((uint64_t)(T.vbase + s) << 32) | (T.vbase + d);
          }
          A.samp[v] = e;
        }
      }
    }
    for (uint32_t k = gwarp; round > 0 && k < nroots; k += gwarps) {
      const uint32_t v = round == 0 ? A.vlo + k : __ldcg(&A.roots[k]);
      const uint32_t t = A.vtenant ? A.vtenant[v] : 0u;
      if (s_done[t]) continue;
      const uint32_t sz = round == 0 ? 1u : __ldcg(&A.size[v]);
      const GsBorTenant& T = tenant_of(A, t);
      const uint32_t col = round == 0 ? T.round0_col : round;
      GsBucket* acc = A.acc + (size_t)v * A.W;
      if (col >= T.ns) {  // OutOfSamplesException
        if (lane == 0) A.tstate[4 * t + 3] = 1u;
      } else {
        const GsBucket* own = A.sk + T.sk_off + (size_t)(v - T.vbase) * T.nb;
        uint32_t code;
        uint64_t idx;
        if (sz > 1) sample_warp(acc, acc + T.bkt, T.bkt, T.csmix, &code, &idx);
        else sample_warp(own + (size_t)col * T.bkt, own + (T.nb - 1), T.bkt, T.csmix, &code, &idx);
        if (lane == 0) {
          uint64_t e = ~0ull;
          if (code == kFail) {
            A.tstate[4 * t + 1] = 1u;
          } else if (code == kGood) {
            const uint32_t s = (uint32_t)(idx >> 32), d = (uint32_t)idx;
            if (s < T.V && d < T.V && s != d)  // anything else is a checksum collision
              e = ((uint64_t)(T.vbase + s) << 32) | (T.vbase + d);
          }
          A.samp[v] = e;
        }
      }
      if (sz > 1) {
        __syncwarp();
        for (uint32_t j = lane; j <= T.bkt; j += 32) acc[j] = GsBucket{0, 0};
      }
    }
    if (!grid_sync(bcount, bgen, err, A.wait_ns)) return;

    // ---- union the sampled edges: one thread per root, so many DSU walks are in flight ----
    for (uint32_t k = gtid; k < nroots; k += gthreads) {
      const uint32_t v = round == 0 ? A.vlo + k : __ldcg(&A.roots[k]);
      const uint32_t t = A.vtenant ? A.vtenant[v] : 0u;
      if (s_done[t]) continue;
      const GsBorTenant& T = tenant_of(A, t);
      if ((round == 0 ? T.round0_col : round) >= T.ns) continue;
      const uint64_t e = __ldcg(&A.samp[v]);
      if (e == ~0ull) continue;
      const uint32_t gs = (uint32_t)(e >> 32), gd = (uint32_t)e;
      if (dsu_union(A.parent, gs, gd, limit, err)) {
        // read before writing: with one graph every successful union (2^17 in round 0 at V=2^17)
        // would store to the same flag, and those stores queue on one L2 line
        if (!ld_volatile(&A.tstate[4 * t + 1])) A.tstate[4 * t + 1] = 1u;
        const uint32_t f = atomicAdd(&A.status[4], 1u);
        if (f < A.forest_cap) {
          A.forest[2 * f] = min(gs, gd);
          A.forest[2 * f + 1] = max(gs, gd);
        }
      }
    }
    if (!grid_sync(bcount, bgen, err, A.wait_ns)) return;

    // ---- compress, clear the sizes and the root list for the next round, and per tenant stop
    //      at the first unmodified round (the modified flags were final at the last barrier) ----
    for (uint32_t v = A.vlo + gtid; v < A.V; v += gthreads) {
      A.parent[v] = dsu_root(A.parent, v, limit, err);
      A.size[v] = 0;
    }
    if (gtid == 0) {
      *nroots_p = 0;
      *acc_next = 0;
    }
    if (A.complement)
      for (uint32_t t = gtid; t < A.T; t += gthreads) A.largest[t] = 0ull;
    for (uint32_t t = gtid; t < A.T; t += gthreads) {
      volatile uint32_t* ts = A.tstate + 4 * t;
      if (ts[0]) continue;
      if (ts[3]) {                     // ran out of samples
        ts[0] = 1u;
        atomicSub(&A.status[5], 1u);
      } else if (ts[1]) {              // modified: the next round runs
        ts[1] = 0u;
        ts[2] = round + 1;
        if (round + 1 >= tenant_of(A, t).ns) {
          ts[3] = 1u;
          ts[0] = 1u;
          atomicSub(&A.status[5], 1u);
        }
      } else {
        ts[0] = 1u;
        atomicSub(&A.status[5], 1u);
      }
    }
    if (!grid_sync(bcount, bgen, err, A.wait_ns)) return;
    if (ld_volatile(&A.status[5]) == 0) return;
  }
}

}  // namespace

gs_status gs_boruvka_launch(const GsBorLaunch& L, cudaStream_t s) {
  BorArgs A;
  A.sk = L.sk;
  A.tenants = L.T > 1 ? L.tenants : nullptr;
  A.t0 = L.t0;
  A.vtenant = L.T > 1 ? L.vtenant : nullptr;
  A.T = L.T;
  A.V = L.V;
  A.W = L.W;
  A.vlo = L.vlo;
  A.max_rounds = L.max_rounds;
  A.parent = L.parent;
  A.size = L.size;
  A.acc = L.acc;
  A.samp = L.samp;
  A.roots = L.roots;
  A.forest = L.forest;
  A.forest_cap = L.forest_cap;
  A.status = L.status;
  A.tstate = L.tstate;
  A.wait_ns = L.wait_ns;
  A.complement = (L.complement && L.largest) ? 1u : 0u;
  A.largest = A.complement ? L.largest : nullptr;
  int dev = 0;
  GS_CUDA_TRY(cudaGetDevice(&dev));
  const size_t smem = (size_t)((L.T + 3u) & ~3u) * sizeof(uint32_t) + (size_t)kWarps * kAccRun * L.W * sizeof(GsBucket);
  // occupancy depends on the shared-memory size: cache it per (device, size)
  struct Occ { size_t smem = 0; int blocks = 0; };
  static thread_local Occ occ[64];  // per host thread: handles may be used from several threads at once
  Occ& o = occ[dev < 64 ? dev : 63];
  if (o.smem != smem) {
    GS_CUDA_TRY(cudaFuncSetAttribute(k_boruvka, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, sms = 0;
    GS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_boruvka, kThreads, smem));
    GS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) {
      gs_set_error("Boruvka kernel does not fit on an SM with " + std::to_string(smem) + " bytes of shared memory");
      return GS_ERR_BAD_ARG;
    }
    o.smem = smem;
    o.blocks = per_sm * sms;  // every block co-resident: the cooperative-launch limit
  }
  // cooperative through a launch attribute, so the launch can also be captured into a CUDA graph
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(o.blocks);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  GS_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_boruvka, A));
  return GS_OK;
}

gs_status gs_boruvka_enqueue(gs_graph* g, uint32_t level, uint32_t round0_col, cudaStream_t s, uint32_t* h_out) {
  const uint32_t V = g->V, nb = g->geom.num_buckets, bkt = g->geom.bkt_per_col;
  g->labels_valid = false;
  g->last_forest_edges = 0;

  GsBorLaunch L;
  L.sk = g->d_sk + (size_t)level * V * nb;
  L.t0.sk_off = 0;
  L.t0.vbase = 0;
  L.t0.V = V;
  L.t0.nb = nb;
  L.t0.bkt = bkt;
  L.t0.ns = g->geom.num_samples;
  L.t0.round0_col = round0_col;
  L.t0.csmix = gs_seed_mix(g->seed);
  L.T = 1;
  L.V = V;
  L.W = bkt + 1;
  L.max_rounds = g->geom.num_samples;
  L.parent = g->d_parent;
  L.size = g->d_size;
  L.acc = g->d_acc;
  L.samp = g->d_samp;
  L.roots = g->d_res;
  L.forest = g->d_forest;
  L.forest_cap = V;
  L.status = g->d_status;
  L.tstate = g->d_status + 8;
  L.wait_ns = g->wait_ns;
  L.complement = g->sketches_symmetric ? 1u : 0u;
  L.largest = reinterpret_cast<unsigned long long*>(g->d_status + 18);   // status words 18-19

  // the kernel expects all-zero accumulator rows and leaves them so when it runs to the end
  if (g->acc_dirty) GS_CUDA_TRY(cudaMemsetAsync(g->d_acc, 0, (size_t)V * (bkt + 1) * sizeof(GsBucket), s));
  g->acc_dirty = true;
  // the ingest error bits not yet reported move to word 16 (read back with the query's words);
  // status: everything else zero except the count of tenants still running
  GS_CUDA_TRY(cudaMemcpyAsync(g->d_status + 16, g->d_status, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  g->h_status[15] = 1;
  GS_CUDA_TRY(cudaMemsetAsync(g->d_status, 0, 16 * sizeof(uint32_t), s));
  GS_CUDA_TRY(cudaMemcpyAsync(g->d_status + 5, g->h_status + 15, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  {
    GsProfScope ps(g, GS_PROF_QUERY, s, 1);
    GS_TRY(gs_boruvka_launch(L, s));
  }
  GS_CUDA_TRY(cudaMemcpyAsync(h_out, g->d_status, 17 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  // the query's error bits are read back with its words: the error word starts clean for the ingest
  // calls queued after the query (a stale bit would fail the next synchronizing call)
  GS_CUDA_TRY(cudaMemsetAsync(g->d_status, 0, sizeof(uint32_t), s));
  return GS_OK;
}

gs_status gs_boruvka_finish(gs_graph* g, uint32_t level, const uint32_t* st) {
  if (st[0] & GS_DEV_ERR_TIMEOUT) {
    gs_set_error("a grid barrier of the Boruvka kernel gave up waiting");
    return GS_ERR_TIMEOUT;
  }
  if (st[0] & GS_DEV_ERR_DSU_LIMIT) {
    gs_set_error("DSU walk exceeded its bound");
    return GS_ERR_INTERNAL;
  }
  g->acc_dirty = false;
  if (st[8 + 3]) {
    gs_set_error("sketch ran out of samples after " + std::to_string(st[8 + 2]) + " Boruvka rounds");
    return GS_ERR_SKETCH_FAIL;
  }
  g->last_rounds = st[8 + 2];
  g->last_forest_edges = st[4] < g->V ? st[4] : g->V - 1;
  g->labels_valid = true;
  g->labels_level = level;
  return GS_OK;
}

gs_status gs_boruvka(gs_graph* g, uint32_t level, uint32_t round0_col, cudaStream_t s) {
  GS_TRY(gs_boruvka_enqueue(g, level, round0_col, s, g->h_status));
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  return gs_boruvka_finish(g, level, g->h_status);
}
