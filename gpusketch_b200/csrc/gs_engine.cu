// gs_engine.cu - many independent connected-components graphs (tenants) on one GPU.
//
// The tenants' sketches live in one device arena (first-fit by bucket range) and every tenant owns
// a run of consecutive ids in the engine's vertex space.  An ingest call carries slices of records
// for many tenants: one kernel rewrites the tenant-local endpoints into the vertex space, then the
// endpoint bucketing and the sketch update of the single-graph path run once over all of them.  The
// sketch-update kernel's tenant variant reads each work chunk's geometry, column constants and
// arena offset from the tenant table, so a tenant's buckets get exactly the XORs a gs_graph with
// the same V, seed and sketches_factor would get (src/cc_sketch_alg.cpp:154-160, src/sketch.cpp:
// 110-131 of the reference).  A query runs the persistent Boruvka kernel over the listed tenants
// in one cooperative launch; the others are marked done before it starts.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "gs_internal.h"

namespace {

struct EngTenant {
  bool live = false;
  uint32_t V = 0;
  uint32_t vbase = 0;
  uint64_t sk_off = 0;   // bucket offset in the arena
  uint64_t buckets = 0;  // V * num_buckets
  uint64_t seed = 0;
  double factor = 1.0;
  GsGeom geom{};
};

// First-fit allocator over [0, capacity) with coalescing frees.
class RangeAlloc {
 public:
  void reset(uint64_t capacity) {
    free_.clear();
    if (capacity) free_[0] = capacity;
  }
  bool alloc(uint64_t n, uint64_t* at) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *at = it->first;
      const uint64_t rest = it->second - n, start = it->first + n;
      free_.erase(it);
      if (rest) free_[start] = rest;
      return true;
    }
    return false;
  }
  void release(uint64_t at, uint64_t n) {
    auto next = free_.lower_bound(at);
    if (next != free_.end() && next->first == at + n) {
      n += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == at) {
        prev->second += n;
        return;
      }
    }
    free_[at] = n;
  }

 private:
  std::map<uint64_t, uint64_t> free_;  // start -> length
};

__global__ void k_fill_u32(uint32_t* __restrict__ p, uint32_t n, uint32_t value) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = value;
}

// Tenant-local records -> engine vertex space.  Record i (absolute index first + i) belongs to the
// slice s with off[s] <= first + i < off[s+1].  Records naming a vertex outside their tenant, or
// a dead tenant, become (~0, ~0): the bucketing skips them and the error word reports them.  in
// and out may be the same buffer (each thread rewrites its own records).
__global__ void k_globalize(const uint2* in, uint2* out, uint64_t first, uint64_t m,
                            const uint64_t* __restrict__ off, const uint32_t* __restrict__ sten, uint32_t ns,
                            const GsIngTenant* __restrict__ ten, uint32_t num_ten, uint32_t* __restrict__ status) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = first + i;
    uint32_t lo = 0, hi = ns;  // largest s with off[s] <= r
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (off[mid] <= r) lo = mid; else hi = mid;
    }
    const uint32_t t = sten[lo];
    const uint2 p = in[i];
    uint2 q = make_uint2(0xffffffffu, 0xffffffffu);
    if (t < num_ten) {
      const GsIngTenant T = ten[t];
      if (T.V != 0 && p.x < T.V && p.y < T.V) q = make_uint2(T.vbase + p.x, T.vbase + p.y);
    }
    if (q.x == 0xffffffffu) atomicOr(status, (uint32_t)GS_DEV_ERR_VERTEX_RANGE);
    out[i] = q;
  }
}

// Local labels of the queried tenants, back to back in query order, and each one's root count.
__global__ void k_gather_labels(const uint32_t* __restrict__ parent, const uint32_t* __restrict__ qten,
                                const uint32_t* __restrict__ qoff, const GsBorTenant* __restrict__ bor,
                                uint32_t* __restrict__ labels, uint32_t* __restrict__ ncc) {
  const uint32_t q = blockIdx.y;
  const GsBorTenant T = bor[qten[q]];
  uint32_t roots = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T.V; i += gridDim.x * blockDim.x) {
    const uint32_t p = parent[T.vbase + i];
    labels[qoff[q] + i] = p - T.vbase;
    roots += p == T.vbase + i;
  }
  for (int o = 16; o > 0; o >>= 1) roots += __shfl_xor_sync(0xffffffffu, roots, o);
  if ((threadIdx.x & 31u) == 0 && roots) atomicAdd(&ncc[q], roots);
}

template <typename T>
gs_status grow_device(T** p, uint64_t* cap, uint64_t want) {
  if (*cap >= want) return GS_OK;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  GS_CUDA_TRY(cudaMalloc(p, want * sizeof(T)));
  *cap = want;
  return GS_OK;
}

template <typename T>
gs_status grow_pinned(T** p, uint64_t* cap, uint64_t want) {
  if (*cap >= want) return GS_OK;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *cap = 0;
  GS_CUDA_TRY(cudaMallocHost(p, want * sizeof(T)));
  *cap = want;
  return GS_OK;
}

}  // namespace

struct gs_engine {
  gs_graph* g = nullptr;  // plumbing: scratch, stream, staging; g->d_sk is the arena
  int device = 0;
  uint64_t arena_buckets = 0;
  uint32_t max_tenants = 0;  // slot max_tenants is the idle slot of unowned vertex ids
  uint32_t max_vertices = 0;
  uint32_t max_tenant_vertices = 0;
  uint32_t W = 0;  // Boruvka accumulator row width: largest bkt_per_col + 1
  RangeAlloc arena, vspace;
  std::vector<EngTenant> ten;
  uint64_t used_bytes = 0;
  uint32_t live = 0;

  GsIngTenant* d_ing = nullptr;  // [max_tenants + 1]
  GsBorTenant* d_bor = nullptr;  // [max_tenants + 1]
  uint32_t* d_vtenant = nullptr; // [max_vertices]
  uint32_t* d_tstate = nullptr;  // [(max_tenants + 1) * 4] Boruvka per-tenant state
  unsigned long long* d_largest = nullptr;  // [max_tenants + 1] largest component of each tenant per round
  uint32_t* h_tstate = nullptr;  // pinned mirror
  uint32_t* d_qstatus = nullptr; // [16] Boruvka status words
  uint32_t* h_qstatus = nullptr; // pinned [16]
  uint32_t* d_q = nullptr;       // [2 * (max_tenants + 1)] query list, then label offsets
  uint32_t* h_q = nullptr;       // pinned mirror
  uint32_t* d_ncc = nullptr;     // [max_tenants + 1]
  // Slice tables (record offsets and tenants) of an ingest, two sets so that one ingest's tables
  // can be staged while the previous ingest's kernels still read theirs.
  struct SliceTables {
    uint64_t* d_off = nullptr;
    uint64_t* h_off = nullptr;  // pinned
    uint32_t* d_ten = nullptr;
    uint32_t* h_ten = nullptr;  // pinned
    uint64_t cap = 0;           // slices the buffers hold
    cudaEvent_t ev_free = nullptr;  // the last kernel reading these tables has finished
  } tabs[2];
  uint64_t tab_next = 0;
  uint64_t stage_next = 0;  // staging slot of the next ingest_slices chunk
  cudaGraphExec_t phase_exec = nullptr;  // the last recorded phase, updated in place per phase
  uint64_t phase_graphs_built = 0;
  uint64_t phase_graph_launches = 0;
};

namespace {

void free_engine(gs_engine* e) {
  if (!e) return;
  if (e->g) gs_free_graph(e->g);
  cudaFree(e->d_ing); cudaFree(e->d_bor); cudaFree(e->d_vtenant); cudaFree(e->d_tstate); cudaFree(e->d_largest);
  cudaFree(e->d_qstatus); cudaFree(e->d_q); cudaFree(e->d_ncc);
  for (auto& tb : e->tabs) {
    cudaFree(tb.d_off); cudaFree(tb.d_ten);
    if (tb.h_off) cudaFreeHost(tb.h_off);
    if (tb.h_ten) cudaFreeHost(tb.h_ten);
    if (tb.ev_free) cudaEventDestroy(tb.ev_free);
  }
  if (e->h_tstate) cudaFreeHost(e->h_tstate);
  if (e->h_qstatus) cudaFreeHost(e->h_qstatus);
  if (e->h_q) cudaFreeHost(e->h_q);
  if (e->phase_exec) cudaGraphExecDestroy(e->phase_exec);
  delete e;
}

#define GS_ENGINE_GUARD(e)                                                \
  GsDeviceGuard _guard((e)->device);                                      \
  if (!_guard.ok) { gs_set_error("cannot select CUDA device"); return GS_ERR_NO_DEVICE; }

bool tenant_ok(const gs_engine* e, uint32_t t) { return t < e->max_tenants && e->ten[t].live; }

// Column count and bucket depth bounds of the live tenants, for the sketch-update launch.
void refresh_bounds(gs_engine* e) {
  uint32_t cols = 1, min_bkt = 0xffffffffu;
  for (const EngTenant& t : e->ten) {
    if (!t.live) continue;
    cols = std::max(cols, t.geom.num_columns);
    min_bkt = std::min(min_bkt, t.geom.bkt_per_col);
  }
  e->g->ten_max_cols = cols;
  e->g->ten_min_bkt = min_bkt == 0xffffffffu ? 64u : min_bkt;
}

gs_status globalize(gs_engine* e, const uint32_t* in, uint32_t* out, uint64_t first, uint64_t m, uint32_t ns,
                    const gs_engine::SliceTables& tb, cudaStream_t s) {
  const uint64_t want = (m + 255) / 256;
  const int grid = (int)std::min<uint64_t>(std::max<uint64_t>(want, 1), (uint64_t)e->g->num_sms * 16);
  {
    GsProfScope ps(e->g, GS_PROF_BUCKET, s, 1);
    k_globalize<<<grid, 256, 0, s>>>(reinterpret_cast<const uint2*>(in), reinterpret_cast<uint2*>(out), first, m,
                                     tb.d_off, tb.d_ten, ns, e->d_ing, e->max_tenants, e->g->d_status);
  }
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

struct QueryPlan {
  std::vector<uint8_t> seen;
  uint32_t vlo = 0xffffffffu, vhi = 0, max_rounds = 0;
  uint64_t total = 0, maxv = 0;
};

gs_status plan_query(const gs_engine* e, const uint32_t* tenants, uint32_t count, QueryPlan* qp) {
  if (count > e->max_tenants) { gs_set_error("engine query: too many tenants"); return GS_ERR_BAD_ARG; }
  qp->seen.assign(e->max_tenants, 0);
  for (uint32_t i = 0; i < count; i++) {
    const uint32_t t = tenants[i];
    if (!tenant_ok(e, t) || qp->seen[t]) {
      gs_set_error("engine query: tenant " + std::to_string(t) + " is not live or listed twice");
      return GS_ERR_BAD_ARG;
    }
    qp->seen[t] = 1;
    const EngTenant& T = e->ten[t];
    qp->vlo = std::min(qp->vlo, T.vbase);
    qp->vhi = std::max(qp->vhi, T.vbase + T.V);
    qp->max_rounds = std::max(qp->max_rounds, T.geom.num_samples);
    qp->total += T.V;
    qp->maxv = std::max<uint64_t>(qp->maxv, T.V);
  }
  return GS_OK;
}

gs_status check_slices(const gs_engine* e, const uint32_t* sten, const uint64_t* soff, uint32_t ns) {
  for (uint32_t i = 0; i < ns; i++) {
    if (soff[i + 1] < soff[i]) {
      gs_set_error("engine ingest: slice offsets must not decrease");
      return GS_ERR_BAD_ARG;
    }
    if (!tenant_ok(e, sten[i])) {
      gs_set_error("engine ingest: slice " + std::to_string(i) + " names tenant " + std::to_string(sten[i]) +
                   ", which is not live");
      return GS_ERR_BAD_ARG;
    }
  }
  return GS_OK;
}

// Host slice tables -> the pinned buffers of `tb` (whose previous reader has finished).
gs_status stage_slices(gs_engine::SliceTables& tb, const uint32_t* sten, const uint64_t* soff, uint32_t ns) {
  if (tb.cap < (uint64_t)ns + 1) {
    cudaFree(tb.d_off); cudaFree(tb.d_ten);
    if (tb.h_off) cudaFreeHost(tb.h_off);
    if (tb.h_ten) cudaFreeHost(tb.h_ten);
    tb.d_off = nullptr; tb.d_ten = nullptr; tb.h_off = nullptr; tb.h_ten = nullptr; tb.cap = 0;
    const uint64_t cap = std::max<uint64_t>(2 * ((uint64_t)ns + 1), 64);
    GS_CUDA_TRY(cudaMalloc(&tb.d_off, cap * sizeof(uint64_t)));
    GS_CUDA_TRY(cudaMalloc(&tb.d_ten, cap * sizeof(uint32_t)));
    GS_CUDA_TRY(cudaMallocHost(&tb.h_off, cap * sizeof(uint64_t)));
    GS_CUDA_TRY(cudaMallocHost(&tb.h_ten, cap * sizeof(uint32_t)));
    tb.cap = cap;
  }
  if (soff) std::memcpy(tb.h_off, soff, ((size_t)ns + 1) * sizeof(uint64_t));
  if (sten) std::memcpy(tb.h_ten, sten, (size_t)ns * sizeof(uint32_t));
  return GS_OK;
}

gs_status copy_slices(const gs_engine::SliceTables& tb, uint32_t ns, cudaStream_t s) {
  GS_CUDA_TRY(cudaMemcpyAsync(tb.d_off, tb.h_off, ((size_t)ns + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  GS_CUDA_TRY(cudaMemcpyAsync(tb.d_ten, tb.h_ten, (size_t)ns * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  return GS_OK;
}

// Queues one multi-tenant Boruvka launch and the read-back of its results into pinned memory.
// The pinned query tables must not be read by queued work any more.
gs_status enqueue_query(gs_engine* e, const QueryPlan& qp, const uint32_t* tenants, uint32_t count, cudaStream_t s) {
  gs_graph* g = e->g;
  const uint32_t T1 = e->max_tenants + 1;
  // every tenant done except the listed ones; the idle slot stays done
  for (uint32_t t = 0; t < T1; t++) {
    e->h_tstate[4 * t] = t < e->max_tenants && qp.seen[t] ? 0u : 1u;
    e->h_tstate[4 * t + 1] = e->h_tstate[4 * t + 2] = e->h_tstate[4 * t + 3] = 0u;
  }
  std::memset(e->h_qstatus, 0, 16 * sizeof(uint32_t));
  e->h_qstatus[5] = count;
  uint32_t off = 0;
  for (uint32_t i = 0; i < count; i++) {
    e->h_q[i] = tenants[i];
    e->h_q[T1 + i] = off;
    off += e->ten[tenants[i]].V;
  }
  if (g->acc_dirty)
    GS_CUDA_TRY(cudaMemsetAsync(g->d_acc, 0, (size_t)e->max_vertices * e->W * sizeof(GsBucket), s));
  g->acc_dirty = true;
  GS_CUDA_TRY(cudaMemcpyAsync(e->d_tstate, e->h_tstate, (size_t)T1 * 4 * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  GS_CUDA_TRY(cudaMemcpyAsync(e->d_qstatus, e->h_qstatus, 16 * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  GS_CUDA_TRY(cudaMemcpyAsync(e->d_q, e->h_q, (size_t)2 * T1 * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  GS_CUDA_TRY(cudaMemsetAsync(e->d_ncc, 0, (size_t)count * sizeof(uint32_t), s));

  GsBorLaunch L;
  L.sk = g->d_sk;
  L.tenants = e->d_bor;
  L.vtenant = e->d_vtenant;
  L.T = T1;
  L.vlo = qp.vlo;
  L.V = qp.vhi;
  L.W = e->W;
  L.max_rounds = qp.max_rounds;
  L.parent = g->d_parent;
  L.size = g->d_size;
  L.acc = g->d_acc;
  L.samp = g->d_samp;
  L.roots = g->d_res;
  L.forest = g->d_forest;
  L.forest_cap = e->max_vertices;
  L.status = e->d_qstatus;
  L.tstate = e->d_tstate;
  // tenants only take edge records, which reach both endpoints: every tenant's sketches XOR to zero
  L.complement = 1;
  L.largest = e->d_largest;
  {
    GsProfScope ps(g, GS_PROF_QUERY, s, 2);
    GS_TRY(gs_boruvka_launch(L, s));
    const dim3 grid((unsigned)std::min<uint64_t>((qp.maxv + 255) / 256, 64), count);
    k_gather_labels<<<grid, 256, 0, s>>>(g->d_parent, e->d_q, e->d_q + T1, e->d_bor, g->d_res, e->d_ncc);
    GS_CUDA_TRY(cudaGetLastError());
  }
  GS_CUDA_TRY(cudaMemcpyAsync(e->h_qstatus, e->d_qstatus, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GS_CUDA_TRY(cudaMemcpyAsync(e->h_tstate, e->d_tstate, (size_t)T1 * 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GS_CUDA_TRY(cudaMemcpyAsync(e->h_q, e->d_ncc, (size_t)count * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GS_CUDA_TRY(cudaMemcpyAsync(g->h_status, g->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  return GS_OK;
}

// After the queued query finished: error words, per-tenant results, labels.
gs_status finish_query(gs_engine* e, const QueryPlan& qp, const uint32_t* tenants, uint32_t count, uint32_t* labels,
                       uint32_t* num_cc, uint32_t* rounds) {
  gs_graph* g = e->g;
  cudaStream_t s = g->stream;
  if (labels) GS_CUDA_TRY(cudaMemcpy(labels, g->d_res, qp.total * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  const uint32_t qerr = e->h_qstatus[0], ierr = g->h_status[0];
  g->acc_dirty = (qerr & (GS_DEV_ERR_TIMEOUT | GS_DEV_ERR_DSU_LIMIT)) != 0;
  if (qerr & GS_DEV_ERR_TIMEOUT) {
    gs_set_error("a grid barrier of the Boruvka kernel gave up waiting");
    return GS_ERR_TIMEOUT;
  }
  if (qerr & GS_DEV_ERR_DSU_LIMIT) {
    gs_set_error("DSU walk exceeded its bound");
    return GS_ERR_INTERNAL;
  }
  std::string oos;
  for (uint32_t i = 0; i < count; i++) {
    const uint32_t* ts = e->h_tstate + 4 * tenants[i];
    if (num_cc) num_cc[i] = e->h_q[i];
    if (rounds) rounds[i] = ts[2];
    if (ts[3]) oos += (oos.empty() ? "" : ", ") + std::to_string(tenants[i]);
  }
  if (ierr) {
    GS_CUDA_TRY(cudaMemsetAsync(g->d_status, 0, sizeof(uint32_t), s));
    GS_CUDA_TRY(cudaStreamSynchronize(s));
    if (ierr & GS_DEV_ERR_VERTEX_RANGE) {
      gs_set_error("an edge record named a vertex id >= its tenant's num_vertices; those records were skipped");
      return GS_ERR_BAD_ARG;
    }
    gs_set_error("device consistency check failed (bits " + std::to_string(ierr) + ")");
    return GS_ERR_INTERNAL;
  }
  if (!oos.empty()) {
    gs_set_error("sketches ran out of samples for tenant(s) " + oos);
    return GS_ERR_SKETCH_FAIL;
  }
  return GS_OK;
}

}  // namespace

extern "C" {

gs_status gs_engine_tenant_bytes(uint32_t num_vertices, double sketches_factor, uint64_t* bytes) {
  if (!bytes || num_vertices < 2) { gs_set_error("gs_engine_tenant_bytes: bad arguments"); return GS_ERR_BAD_ARG; }
  const GsGeom geom = gs_make_geom(num_vertices, sketches_factor > 0 ? sketches_factor : 1.0);
  *bytes = (uint64_t)num_vertices * geom.num_buckets * sizeof(GsBucket);
  return GS_OK;
}

gs_status gs_engine_create(const gs_engine_config* cfg, gs_engine** out) {
  if (!cfg || !out) { gs_set_error("gs_engine_create: null argument"); return GS_ERR_BAD_ARG; }
  *out = nullptr;
  if (cfg->max_tenants < 1 || cfg->max_tenants > 4096 || cfg->max_vertices < 2 ||
      cfg->max_vertices >= 0xffffffffu - 64 || cfg->max_tenant_vertices < 2 ||
      cfg->max_tenant_vertices > cfg->max_vertices || cfg->sketch_budget_bytes < sizeof(GsBucket)) {
    gs_set_error("gs_engine_create: need 1 <= max_tenants <= 4096, 2 <= max_tenant_vertices <= max_vertices < 2^32 - 64 "
                 "and a sketch budget");
    return GS_ERR_BAD_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    gs_set_error("no CUDA device");
    return GS_ERR_NO_DEVICE;
  }
  int dev = cfg->device;
  if (dev < 0) cudaGetDevice(&dev);
  if (dev >= ndev) { gs_set_error("device ordinal out of range"); return GS_ERR_BAD_ARG; }
  GsDeviceGuard guard(dev);
  if (!guard.ok) { gs_set_error("cannot select CUDA device"); return GS_ERR_NO_DEVICE; }

  std::unique_ptr<gs_engine, void (*)(gs_engine*)> e(new gs_engine(), free_engine);
  e->device = dev;
  e->max_tenants = cfg->max_tenants;
  e->max_vertices = cfg->max_vertices;
  e->max_tenant_vertices = cfg->max_tenant_vertices;
  e->arena_buckets = cfg->sketch_budget_bytes / sizeof(GsBucket);
  e->arena.reset(e->arena_buckets);
  e->vspace.reset(e->max_vertices);
  e->ten.resize(e->max_tenants);
  const GsGeom big = gs_make_geom(e->max_tenant_vertices, 1.0);
  e->W = big.bkt_per_col + 1;

  // the plumbing handle: one level over the whole vertex space, the arena as its sketches
  e->g = new gs_graph();
  gs_graph* g = e->g;
  g->V = e->max_vertices;
  g->num_levels = 1;
  g->num_subgraphs = 1;
  g->device = dev;
  g->geom = big;
  g->max_batch_edges = cfg->max_batch_edges ? std::min<uint64_t>(cfg->max_batch_edges, 1ull << 30) : (1ull << 25);
  cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, dev);
  g->tune = gs_tune_for(big, g->num_sms);
  g->sample_cursor.assign(1, 0);
  GS_CUDA_TRY(cudaStreamCreateWithFlags(&g->own_stream, cudaStreamNonBlocking));
  g->stream = g->own_stream;
  GS_CUDA_TRY(cudaEventCreateWithFlags(&g->ev_order, cudaEventDisableTiming));
  if (cudaMalloc(&g->d_sk, e->arena_buckets * sizeof(GsBucket)) != cudaSuccess) {
    cudaGetLastError();
    gs_set_error("gs_engine_create: cannot allocate a sketch arena of " + std::to_string(cfg->sketch_budget_bytes) +
                 " bytes");
    return GS_ERR_OOM;
  }
  const uint32_t T1 = e->max_tenants + 1;
  GS_CUDA_TRY(cudaMalloc(&g->d_colmix, (size_t)T1 * kColStride * sizeof(uint64_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_status, 32 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMemsetAsync(g->d_status, 0, 32 * sizeof(uint32_t), g->stream));
  GS_CUDA_TRY(cudaMallocHost(&g->h_status, 32 * sizeof(uint32_t)));
  const size_t V = e->max_vertices;
  GS_CUDA_TRY(cudaMalloc(&g->d_parent, V * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_size, V * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_res, V * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_samp, V * sizeof(uint64_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_acc, V * e->W * sizeof(GsBucket)));
  GS_CUDA_TRY(cudaMalloc(&g->d_forest, 2 * V * sizeof(uint32_t)));

  GS_CUDA_TRY(cudaMalloc(&e->d_ing, (size_t)T1 * sizeof(GsIngTenant)));
  GS_CUDA_TRY(cudaMalloc(&e->d_bor, (size_t)T1 * sizeof(GsBorTenant)));
  GS_CUDA_TRY(cudaMalloc(&e->d_largest, (size_t)T1 * sizeof(unsigned long long)));
  GS_CUDA_TRY(cudaMemsetAsync(e->d_ing, 0, (size_t)T1 * sizeof(GsIngTenant), g->stream));
  GS_CUDA_TRY(cudaMemsetAsync(e->d_bor, 0, (size_t)T1 * sizeof(GsBorTenant), g->stream));
  GS_CUDA_TRY(cudaMalloc(&e->d_vtenant, V * sizeof(uint32_t)));
  k_fill_u32<<<g->num_sms * 4, 256, 0, g->stream>>>(e->d_vtenant, (uint32_t)V, e->max_tenants);
  GS_CUDA_TRY(cudaGetLastError());
  GS_CUDA_TRY(cudaMalloc(&e->d_tstate, (size_t)T1 * 4 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMallocHost(&e->h_tstate, (size_t)T1 * 4 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&e->d_qstatus, 32 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMallocHost(&e->h_qstatus, 16 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&e->d_q, (size_t)2 * T1 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMallocHost(&e->h_q, (size_t)2 * T1 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&e->d_ncc, (size_t)T1 * sizeof(uint32_t)));
  for (auto& tb : e->tabs) GS_CUDA_TRY(cudaEventCreateWithFlags(&tb.ev_free, cudaEventDisableTiming));
  g->d_vtenant = e->d_vtenant;
  g->d_ten = e->d_ing;
  refresh_bounds(e.get());
  // staging and bucketing scratch for a full batch are allocated now, so that serving allocates
  // nothing once it has started
  GS_TRY(gs_ensure_pair_staging(g));
  GS_TRY(gs_reserve_ingest(g, g->max_batch_edges));
  GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  *out = e.release();
  return GS_OK;
}

gs_status gs_engine_destroy(gs_engine* e) {
  if (!e) return GS_OK;
  GsDeviceGuard guard(e->device);
  if (e->g && e->g->stream) cudaStreamSynchronize(e->g->stream);
  free_engine(e);
  return GS_OK;
}

gs_status gs_engine_add_tenant(gs_engine* e, uint32_t num_vertices, uint64_t seed, double sketches_factor,
                               uint32_t* tenant) {
  if (!e || !tenant) { gs_set_error("gs_engine_add_tenant: null argument"); return GS_ERR_BAD_ARG; }
  if (num_vertices < 2 || num_vertices > e->max_tenant_vertices) {
    gs_set_error("gs_engine_add_tenant: num_vertices must be in [2, max_tenant_vertices = " +
                 std::to_string(e->max_tenant_vertices) + "]");
    return GS_ERR_BAD_ARG;
  }
  const double factor = sketches_factor > 0 ? sketches_factor : 1.0;
  const GsGeom geom = gs_make_geom(num_vertices, factor);
  if (geom.num_columns > 64 || geom.num_columns + 1 > kColStride) {
    gs_set_error("gs_engine_add_tenant: more than 64 sketch columns are not supported");
    return GS_ERR_BAD_ARG;
  }
  GS_ENGINE_GUARD(e);
  uint32_t slot = e->max_tenants;
  for (uint32_t t = 0; t < e->max_tenants; t++)
    if (!e->ten[t].live) { slot = t; break; }
  if (slot == e->max_tenants) {
    gs_set_error("gs_engine_add_tenant: not admitted, all " + std::to_string(e->max_tenants) + " tenant slots in use");
    return GS_ERR_OOM;
  }
  const uint64_t buckets = (uint64_t)num_vertices * geom.num_buckets;
  uint64_t sk_off = 0, vbase = 0;
  if (!e->arena.alloc(buckets, &sk_off)) {
    gs_set_error("gs_engine_add_tenant: not admitted, " + std::to_string(buckets * sizeof(GsBucket)) +
                 " sketch bytes do not fit in the arena (" + std::to_string(e->used_bytes) + " of " +
                 std::to_string(e->arena_buckets * sizeof(GsBucket)) + " in use)");
    return GS_ERR_OOM;
  }
  if (!e->vspace.alloc(num_vertices, &vbase)) {
    e->arena.release(sk_off, buckets);
    gs_set_error("gs_engine_add_tenant: not admitted, no run of " + std::to_string(num_vertices) +
                 " free ids in the engine vertex space");
    return GS_ERR_OOM;
  }
  EngTenant& T = e->ten[slot];
  T.live = true;
  T.V = num_vertices;
  T.vbase = (uint32_t)vbase;
  T.sk_off = sk_off;
  T.buckets = buckets;
  T.seed = seed;
  T.factor = factor;
  T.geom = geom;

  gs_graph* g = e->g;
  cudaStream_t s = g->stream;
  GsIngTenant it{};
  it.sk_off = sk_off;
  it.vbase = T.vbase;
  it.V = num_vertices;
  it.C = geom.num_columns;
  it.bkt = geom.bkt_per_col;
  it.nb = geom.num_buckets;
  GsBorTenant bt{};
  bt.sk_off = sk_off;
  bt.csmix = gs_seed_mix(seed);
  bt.vbase = T.vbase;
  bt.V = num_vertices;
  bt.nb = geom.num_buckets;
  bt.bkt = geom.bkt_per_col;
  bt.ns = geom.num_samples;
  bt.round0_col = 0;
  std::vector<uint64_t> colmix(kColStride, 0);
  for (uint32_t c = 0; c < geom.num_columns; c++) colmix[c] = gs_seed_mix(seed + 5ull * c);  // column_seed (sketch.h:303)
  colmix[geom.num_columns] = gs_seed_mix(seed);                                               // checksum_seed (sketch.h:304)
  // pageable sources: each copy is staged before the call returns, in stream order
  GS_CUDA_TRY(cudaMemsetAsync(g->d_sk + sk_off, 0, buckets * sizeof(GsBucket), s));
  GS_CUDA_TRY(cudaMemcpyAsync(g->d_colmix + (size_t)slot * kColStride, colmix.data(), kColStride * sizeof(uint64_t),
                              cudaMemcpyHostToDevice, s));
  GS_CUDA_TRY(cudaMemcpyAsync(e->d_ing + slot, &it, sizeof(it), cudaMemcpyHostToDevice, s));
  GS_CUDA_TRY(cudaMemcpyAsync(e->d_bor + slot, &bt, sizeof(bt), cudaMemcpyHostToDevice, s));
  k_fill_u32<<<(num_vertices + 255) / 256, 256, 0, s>>>(e->d_vtenant + T.vbase, num_vertices, slot);
  GS_CUDA_TRY(cudaGetLastError());
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  e->used_bytes += buckets * sizeof(GsBucket);
  e->live++;
  refresh_bounds(e);
  *tenant = slot;
  return GS_OK;
}

gs_status gs_engine_remove_tenant(gs_engine* e, uint32_t tenant) {
  if (!e) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  if (!tenant_ok(e, tenant)) { gs_set_error("gs_engine_remove_tenant: no such tenant"); return GS_ERR_BAD_ARG; }
  GS_ENGINE_GUARD(e);
  gs_graph* g = e->g;
  cudaStream_t s = g->stream;
  EngTenant& T = e->ten[tenant];
  // queued ingests of this tenant finish before its ids and arena range can be handed out again
  const GsIngTenant dead{};
  const GsBorTenant dead_b{};
  GS_CUDA_TRY(cudaMemcpyAsync(e->d_ing + tenant, &dead, sizeof(dead), cudaMemcpyHostToDevice, s));
  GS_CUDA_TRY(cudaMemcpyAsync(e->d_bor + tenant, &dead_b, sizeof(dead_b), cudaMemcpyHostToDevice, s));
  k_fill_u32<<<(T.V + 255) / 256, 256, 0, s>>>(e->d_vtenant + T.vbase, T.V, e->max_tenants);
  GS_CUDA_TRY(cudaGetLastError());
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  e->arena.release(T.sk_off, T.buckets);
  e->vspace.release(T.vbase, T.V);
  e->used_bytes -= T.buckets * sizeof(GsBucket);
  e->live--;
  T = EngTenant{};
  refresh_bounds(e);
  return GS_OK;
}

gs_status gs_engine_clear_tenant(gs_engine* e, uint32_t tenant) {
  if (!e || !tenant_ok(e, tenant)) { gs_set_error("gs_engine_clear_tenant: no such tenant"); return GS_ERR_BAD_ARG; }
  GS_ENGINE_GUARD(e);
  const EngTenant& T = e->ten[tenant];
  GS_CUDA_TRY(cudaMemsetAsync(e->g->d_sk + T.sk_off, 0, T.buckets * sizeof(GsBucket), e->g->stream));
  return GS_OK;
}

gs_status gs_engine_memory(const gs_engine* e, uint64_t* used, uint64_t* capacity, uint32_t* live_tenants) {
  if (!e) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  if (used) *used = e->used_bytes;
  if (capacity) *capacity = e->arena_buckets * sizeof(GsBucket);
  if (live_tenants) *live_tenants = e->live;
  return GS_OK;
}

gs_status gs_engine_set_stream(gs_engine* e, void* stream) {
  if (!e) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  return gs_graph_set_stream(e->g, stream);
}

gs_status gs_engine_ingest(gs_engine* e, const uint32_t* slice_tenants, const uint64_t* slice_offsets,
                           uint32_t num_slices, const uint32_t* pairs, int pairs_on_device, void* stream) {
  if (!e || (num_slices && (!slice_tenants || !slice_offsets))) {
    gs_set_error("gs_engine_ingest: null argument");
    return GS_ERR_BAD_ARG;
  }
  if (num_slices == 0) return GS_OK;
  GS_TRY(check_slices(e, slice_tenants, slice_offsets, num_slices));
  const uint64_t first = slice_offsets[0], n = slice_offsets[num_slices] - first;
  if (n == 0) return GS_OK;
  if (!pairs) { gs_set_error("gs_engine_ingest: null pairs"); return GS_ERR_BAD_ARG; }
  GS_ENGINE_GUARD(e);
  gs_graph* g = e->g;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g->stream;
  g->labels_valid = false;
  GS_TRY(gs_ensure_pair_staging(g));
  gs_engine::SliceTables& tb = e->tabs[e->tab_next++ & 1];
  GS_CUDA_TRY(cudaEventSynchronize(tb.ev_free));
  GS_TRY(stage_slices(tb, slice_tenants, slice_offsets, num_slices));
  GS_TRY(copy_slices(tb, num_slices, s));
  const uint64_t cap = g->pairs_cap;

  cudaPointerAttributes attr{};
  const bool pinned = !pairs_on_device && cudaPointerGetAttributes(&attr, pairs) == cudaSuccess &&
                      attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  uint32_t* hp = static_cast<uint32_t*>(g->h_pin);
  for (uint64_t done = 0, k = 0; done < n; k++) {
    const uint64_t m = std::min(cap, n - done);
    const int slot = (int)(k & 1);
    uint32_t* dslot = g->d_pairs + (size_t)slot * cap * 2;
    // the slice two steps back used this slot; it must be consumed before the slot is rewritten
    GS_CUDA_TRY(cudaEventSynchronize(g->ev_done[slot]));
    const uint32_t* src = pairs + 2 * (first + done);
    if (pairs_on_device) {
      GS_TRY(globalize(e, src, dslot, first + done, m, num_slices, tb, s));
    } else {
      if (!pinned) {
        std::memcpy(hp + (size_t)slot * cap * 2, src, (size_t)m * 2 * sizeof(uint32_t));
        src = hp + (size_t)slot * cap * 2;
      }
      GS_CUDA_TRY(cudaMemcpyAsync(dslot, src, (size_t)m * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, g->copy_stream));
      GS_CUDA_TRY(cudaEventRecord(g->ev_copy[slot], g->copy_stream));
      GS_CUDA_TRY(cudaStreamWaitEvent(s, g->ev_copy[slot], 0));
      GS_TRY(globalize(e, dslot, dslot, first + done, m, num_slices, tb, s));
    }
    GS_TRY(gs_ingest_device_pairs(g, dslot, m, -1, s));
    GS_CUDA_TRY(cudaEventRecord(g->ev_done[slot], s));
    done += m;
  }
  GS_CUDA_TRY(cudaEventRecord(tb.ev_free, s));
  if (!pairs_on_device) GS_CUDA_TRY(cudaStreamSynchronize(g->copy_stream));
  if (s != g->stream) {
    GS_CUDA_TRY(cudaEventRecord(g->ev_order, s));
    GS_CUDA_TRY(cudaStreamWaitEvent(g->stream, g->ev_order, 0));
  }
  return GS_OK;
}

gs_status gs_engine_ingest_slices(gs_engine* e, uint32_t num_slices, const uint32_t* slice_tenants,
                                  const uint64_t* slice_counts, const uint32_t* const* slice_pairs, void* stream) {
  if (!e || (num_slices && (!slice_tenants || !slice_counts || !slice_pairs))) {
    gs_set_error("gs_engine_ingest_slices: null argument");
    return GS_ERR_BAD_ARG;
  }
  uint64_t total = 0;
  for (uint32_t i = 0; i < num_slices; i++) {
    if (!tenant_ok(e, slice_tenants[i])) {
      gs_set_error("gs_engine_ingest_slices: slice " + std::to_string(i) + " names tenant " +
                   std::to_string(slice_tenants[i]) + ", which is not live");
      return GS_ERR_BAD_ARG;
    }
    if (slice_counts[i] && !slice_pairs[i]) {
      gs_set_error("gs_engine_ingest_slices: null records of slice " + std::to_string(i));
      return GS_ERR_BAD_ARG;
    }
    total += slice_counts[i];
  }
  if (total == 0) return GS_OK;
  GS_ENGINE_GUARD(e);
  gs_graph* g = e->g;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g->stream;
  g->labels_valid = false;
  GS_TRY(gs_ensure_pair_staging(g));
  const uint64_t cap = g->pairs_cap;
  uint32_t* hp = static_cast<uint32_t*>(g->h_pin);
  bool direct = false;  // some slice was copied straight from caller memory
  uint32_t si = 0;
  uint64_t so = 0;  // records of slice si already staged
  while (si < num_slices) {
    // one staging chunk: whole slices (the last one possibly split) up to `cap` records
    const int slot = (int)(e->stage_next++ & 1);
    gs_engine::SliceTables& tb = e->tabs[slot];
    GS_CUDA_TRY(cudaEventSynchronize(g->ev_done[slot]));
    GS_CUDA_TRY(cudaEventSynchronize(tb.ev_free));
    uint32_t* dslot = g->d_pairs + (size_t)slot * cap * 2;
    uint32_t* hslot = hp + (size_t)slot * cap * 2;
    uint64_t m = 0;
    uint32_t np = 0;
    std::vector<uint64_t> offs{0};
    std::vector<uint32_t> tens;
    while (si < num_slices && m < cap) {
      const uint64_t take = std::min(slice_counts[si] - so, cap - m);
      if (take) {
        const uint32_t* src = slice_pairs[si] + 2 * so;
        cudaPointerAttributes attr{};
        const bool pinned = cudaPointerGetAttributes(&attr, src) == cudaSuccess && attr.type == cudaMemoryTypeHost;
        cudaGetLastError();
        if (!pinned) {
          std::memcpy(hslot + 2 * m, src, (size_t)take * 2 * sizeof(uint32_t));
          src = hslot + 2 * m;
        } else {
          direct = true;
        }
        GS_CUDA_TRY(cudaMemcpyAsync(dslot + 2 * m, src, (size_t)take * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                    g->copy_stream));
        tens.push_back(slice_tenants[si]);
        m += take;
        offs.push_back(m);
        np++;
      }
      so += take;
      if (so == slice_counts[si]) { si++; so = 0; }
    }
    if (np == 0) continue;
    GS_TRY(stage_slices(tb, tens.data(), offs.data(), np));
    GS_TRY(copy_slices(tb, np, g->copy_stream));
    GS_CUDA_TRY(cudaEventRecord(g->ev_copy[slot], g->copy_stream));
    GS_CUDA_TRY(cudaStreamWaitEvent(s, g->ev_copy[slot], 0));
    GS_TRY(globalize(e, dslot, dslot, 0, m, np, tb, s));
    GS_TRY(gs_ingest_device_pairs(g, dslot, m, -1, s));
    GS_CUDA_TRY(cudaEventRecord(g->ev_done[slot], s));
    GS_CUDA_TRY(cudaEventRecord(tb.ev_free, s));
  }
  // caller memory read in place must have landed before the caller may reuse it
  if (direct) GS_CUDA_TRY(cudaStreamSynchronize(g->copy_stream));
  if (s != g->stream) {
    GS_CUDA_TRY(cudaEventRecord(g->ev_order, s));
    GS_CUDA_TRY(cudaStreamWaitEvent(g->stream, g->ev_order, 0));
  }
  return GS_OK;
}

gs_status gs_engine_synchronize(gs_engine* e) {
  if (!e) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  GS_ENGINE_GUARD(e);
  gs_graph* g = e->g;
  GS_CUDA_TRY(cudaMemcpyAsync(g->h_status, g->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
  GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  const uint32_t bits = g->h_status[0];
  if (bits) {
    GS_CUDA_TRY(cudaMemsetAsync(g->d_status, 0, sizeof(uint32_t), g->stream));
    GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if (bits & GS_DEV_ERR_VERTEX_RANGE) {
      gs_set_error("an edge record named a vertex id >= its tenant's num_vertices; those records were skipped");
      return GS_ERR_BAD_ARG;
    }
    gs_set_error("device consistency check failed (bits " + std::to_string(bits) + ")");
    return GS_ERR_INTERNAL;
  }
  return GS_OK;
}

gs_status gs_engine_connected_components(gs_engine* e, const uint32_t* tenants, uint32_t count, uint32_t* labels,
                                         uint32_t* num_cc, uint32_t* rounds) {
  if (!e || (count && !tenants)) { gs_set_error("gs_engine_connected_components: null argument"); return GS_ERR_BAD_ARG; }
  if (count == 0) return GS_OK;
  QueryPlan qp;
  GS_TRY(plan_query(e, tenants, count, &qp));
  GS_ENGINE_GUARD(e);
  gs_graph* g = e->g;
  cudaStream_t s = g->stream;
  GS_TRY(enqueue_query(e, qp, tenants, count, s));
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  return finish_query(e, qp, tenants, count, labels, num_cc, rounds);
}

gs_status gs_engine_phase(gs_engine* e, const uint32_t* slice_tenants, const uint64_t* slice_offsets,
                          uint32_t num_slices, const uint32_t* pairs, const uint32_t* query_tenants,
                          uint32_t query_count, uint32_t* num_cc, uint32_t* rounds, int flags) {
  if (!e || (num_slices && (!slice_tenants || !slice_offsets || !pairs)) || (query_count && !query_tenants)) {
    gs_set_error("gs_engine_phase: null argument");
    return GS_ERR_BAD_ARG;
  }
  GS_TRY(check_slices(e, slice_tenants, slice_offsets, num_slices));
  const uint64_t first = num_slices ? slice_offsets[0] : 0;
  const uint64_t n = num_slices ? slice_offsets[num_slices] - first : 0;
  QueryPlan qp;
  if (query_count) GS_TRY(plan_query(e, query_tenants, query_count, &qp));
  GS_ENGINE_GUARD(e);
  gs_graph* g = e->g;
  cudaStream_t s = g->stream;
  GS_TRY(gs_ensure_pair_staging(g));
  if (n > g->pairs_cap) {
    gs_set_error("gs_engine_phase: at most " + std::to_string(g->pairs_cap) + " records per phase, got " +
                 std::to_string(n));
    return GS_ERR_BAD_ARG;
  }
  // everything the recorded work touches exists before recording starts, and nothing queued on the
  // handle's stream still reads the pinned tables or the staging slot
  GS_TRY(gs_reserve_ingest(g, n));
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  gs_engine::SliceTables& tb = e->tabs[0];
  if (n) GS_TRY(stage_slices(tb, slice_tenants, slice_offsets, num_slices));
  g->labels_valid = false;
  const bool graph = (flags & GS_PHASE_CUDA_GRAPH) != 0;
  if (graph) {
    GS_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    g->capturing = true;
  }
  gs_status st = GS_OK;
  if (n) {
    st = copy_slices(tb, num_slices, s);
    if (st == GS_OK) st = globalize(e, pairs + 2 * first, g->d_pairs, first, n, num_slices, tb, s);
    if (st == GS_OK) st = gs_ingest_device_pairs(g, g->d_pairs, n, -1, s);
  }
  if (st == GS_OK && query_count) st = enqueue_query(e, qp, query_tenants, query_count, s);
  if (graph) {
    g->capturing = false;
    cudaGraph_t cg = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &cg);
    if (st == GS_OK && ce != cudaSuccess) {
      gs_set_error(std::string("gs_engine_phase: stream capture failed: ") + cudaGetErrorString(ce));
      st = GS_ERR_CUDA;
    }
    if (st == GS_OK) {
      // same node sequence as the last phase: update the instantiated graph's parameters in place
      bool updated = false;
      if (e->phase_exec) {
        cudaGraphExecUpdateResultInfo info{};
        updated = cudaGraphExecUpdate(e->phase_exec, cg, &info) == cudaSuccess;
        if (!updated) {
          cudaGetLastError();
          cudaGraphExecDestroy(e->phase_exec);
          e->phase_exec = nullptr;
        }
      }
      if (!updated) {
        const cudaError_t ie = cudaGraphInstantiate(&e->phase_exec, cg, 0);
        if (ie != cudaSuccess) {
          e->phase_exec = nullptr;
          gs_set_error(std::string("gs_engine_phase: graph instantiation failed: ") + cudaGetErrorString(ie));
          st = GS_ERR_CUDA;
        } else {
          e->phase_graphs_built++;
        }
      }
      if (st == GS_OK) {
        const cudaError_t le = cudaGraphLaunch(e->phase_exec, s);
        if (le != cudaSuccess) {
          gs_set_error(std::string("gs_engine_phase: graph launch failed: ") + cudaGetErrorString(le));
          st = GS_ERR_CUDA;
        } else {
          e->phase_graph_launches++;
        }
      }
    }
    if (cg) cudaGraphDestroy(cg);
  }
  GS_TRY(st);
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  if (query_count) return finish_query(e, qp, query_tenants, query_count, nullptr, num_cc, rounds);
  return gs_engine_synchronize(e);
}

gs_status gs_engine_graph_stats(const gs_engine* e, uint64_t* graphs_built, uint64_t* graph_launches) {
  if (!e) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  if (graphs_built) *graphs_built = e->phase_graphs_built;
  if (graph_launches) *graph_launches = e->phase_graph_launches;
  return GS_OK;
}

gs_status gs_engine_tenant_geometry(const gs_engine* e, uint32_t tenant, gs_geometry* out) {
  if (!e || !out || !tenant_ok(e, tenant)) { gs_set_error("gs_engine_tenant_geometry: bad arguments"); return GS_ERR_BAD_ARG; }
  const EngTenant& T = e->ten[tenant];
  out->num_vertices = T.V;
  out->num_samples = T.geom.num_samples;
  out->cols_per_sample = 1;
  out->num_columns = T.geom.num_columns;
  out->bkt_per_col = T.geom.bkt_per_col;
  out->num_buckets = T.geom.num_buckets;
  out->bytes_per_vertex = (uint64_t)T.geom.num_buckets * sizeof(GsBucket);
  return GS_OK;
}

gs_status gs_engine_download_sketches(gs_engine* e, uint32_t tenant, uint32_t first, uint32_t count, gs_bucket* out) {
  if (!e || !out || !tenant_ok(e, tenant) || (uint64_t)first + count > e->ten[tenant].V) {
    gs_set_error("gs_engine_download_sketches: bad arguments");
    return GS_ERR_BAD_ARG;
  }
  GS_ENGINE_GUARD(e);
  const EngTenant& T = e->ten[tenant];
  GS_CUDA_TRY(cudaStreamSynchronize(e->g->stream));
  const size_t nb = T.geom.num_buckets;
  GS_CUDA_TRY(cudaMemcpy(out, e->g->d_sk + T.sk_off + (size_t)first * nb, (size_t)count * nb * sizeof(GsBucket),
                         cudaMemcpyDeviceToHost));
  return GS_OK;
}

gs_status gs_engine_write_binary(gs_engine* e, uint32_t tenant, const char* path) {
  if (!e || !path || !tenant_ok(e, tenant)) { gs_set_error("gs_engine_write_binary: bad arguments"); return GS_ERR_BAD_ARG; }
  const EngTenant& T = e->ten[tenant];
  FILE* f = std::fopen(path, "wb");
  if (!f) { gs_set_error(std::string("cannot open ") + path); return GS_ERR_IO; }
  // header of CCSketchAlg::write_binary (src/cc_sketch_alg.cpp:57-91): seed, V, sketches_factor
  bool ok = std::fwrite(&T.seed, 8, 1, f) == 1 && std::fwrite(&T.V, 4, 1, f) == 1 && std::fwrite(&T.factor, 8, 1, f) == 1;
  const size_t nb = T.geom.num_buckets;
  const uint32_t step = (uint32_t)std::max<size_t>(1, (64u << 20) / (nb * sizeof(GsBucket)));
  std::vector<gs_bucket> buf((size_t)step * nb);
  for (uint32_t v = 0; ok && v < T.V; v += step) {
    const uint32_t c = std::min(step, T.V - v);
    const gs_status st = gs_engine_download_sketches(e, tenant, v, c, buf.data());
    if (st != GS_OK) { std::fclose(f); return st; }
    ok = std::fwrite(buf.data(), sizeof(gs_bucket), (size_t)c * nb, f) == (size_t)c * nb;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { gs_set_error(std::string("write failed: ") + path); return GS_ERR_IO; }
  return GS_OK;
}

gs_status gs_engine_get_tuning(const gs_engine* e, gs_tuning* out) {
  if (!e) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  return gs_get_tuning(e->g, out);
}

gs_status gs_engine_set_tuning(gs_engine* e, const gs_tuning* t) {
  if (!e) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  return gs_set_tuning(e->g, t);
}

gs_status gs_engine_profile_enable(gs_engine* e, int enable) {
  if (!e) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  return gs_profile_enable(e->g, enable);
}

gs_status gs_engine_profile_read(gs_engine* e, gs_profile* out) {
  if (!e) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  return gs_profile_read(e->g, out);
}

}  // extern "C"
