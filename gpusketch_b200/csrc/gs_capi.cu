// gs_capi.cu - the extern "C" boundary declared in include/gpusketch.h.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "gs_internal.h"

namespace {

using DeviceGuard = GsDeviceGuard;

#define GS_GUARD(g)                                                       \
  DeviceGuard _guard((g)->device);                                        \
  if (!_guard.ok) { gs_set_error("cannot select CUDA device"); return GS_ERR_NO_DEVICE; }

cudaStream_t pick_stream(gs_graph* g, void* s) { return s ? static_cast<cudaStream_t>(s) : g->stream; }

}  // namespace

void gs_free_graph(gs_graph* g) {
  if (!g) return;
  cudaFree(g->d_sk); cudaFree(g->d_colmix);
  cudaFree(g->d_cnt); cudaFree(g->d_off); cudaFree(g->d_choff); cudaFree(g->d_tile);
  cudaFree(g->d_nbr); cudaFree(g->d_pairs); cudaFree(g->d_file_pairs); cudaFree(g->d_part); cudaFree(g->d_bkt); cudaFree(g->d_blockhist); cudaFree(g->d_chunkhist); cudaFree(g->d_owner);
  if (g->h_pin) cudaFreeHost(g->h_pin);
  if (g->h_status) cudaFreeHost(g->h_status);
  if (g->h_qstatus) cudaFreeHost(g->h_qstatus);
  if (g->h_qlabels) cudaFreeHost(g->h_qlabels);
  if (g->ev_query) cudaEventDestroy(g->ev_query);
  cudaFree(g->d_status);
  cudaFree(g->d_parent); cudaFree(g->d_size); cudaFree(g->d_res); cudaFree(g->d_samp); cudaFree(g->d_acc);
  cudaFree(g->d_forest);
  cudaFree(g->d_store);
  cudaFree(g->d_store_list);
  cudaFree(g->d_store_status);
  if (g->h_store) cudaFreeHost(g->h_store);
  cudaFree(g->d_eager_set);
  cudaFree(g->d_eager_status);
  if (g->h_eager) cudaFreeHost(g->h_eager);
  for (int i = 0; i < 2; i++) {
    if (g->ev_copy[i]) cudaEventDestroy(g->ev_copy[i]);
    if (g->ev_done[i]) cudaEventDestroy(g->ev_done[i]);
  }
  if (g->copy_stream) cudaStreamDestroy(g->copy_stream);
  if (g->ev_order) cudaEventDestroy(g->ev_order);
  if (g->own_stream) cudaStreamDestroy(g->own_stream);
  delete g;
}

namespace {

// Checks and clears the device error word after the queued work finished.
gs_status check_status(gs_graph* g, cudaStream_t s) {
  GS_CUDA_TRY(cudaMemcpyAsync(g->h_status, g->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  const uint32_t bits = g->h_status[0];
  if (bits) {
    GS_CUDA_TRY(cudaMemsetAsync(g->d_status, 0, sizeof(uint32_t), s));
    GS_CUDA_TRY(cudaStreamSynchronize(s));
    if (bits & GS_DEV_ERR_VERTEX_RANGE) {
      gs_set_error("an edge record named a vertex id >= num_vertices; those records were skipped");
      return GS_ERR_BAD_ARG;
    }
    if (bits & GS_DEV_ERR_TIMEOUT) {
      gs_set_error("a bounded device-side wait gave up");
      return GS_ERR_TIMEOUT;
    }
    gs_set_error("device consistency check failed (bits " + std::to_string(bits) + ")");
    return GS_ERR_INTERNAL;
  }
  return GS_OK;
}

// work queued on a caller stream s must finish before the handle's own stream touches the sketches
gs_status order_after(gs_graph* g, cudaStream_t s) {
  if (s == g->stream) return GS_OK;
  GS_CUDA_TRY(cudaEventRecord(g->ev_order, s));
  GS_CUDA_TRY(cudaStreamWaitEvent(g->stream, g->ev_order, 0));
  return GS_OK;
}

// Host input moves in slices of at most 2^24 pairs.  Per phase the first copy and the last slice's
// ingest overlap nothing and every slice carries a fixed ingest cost (about 0.5 ms at V = 2^17);
// 2^24 balances the two (1 GiB phases: 202.6 ms per 8 phases at 2^25, 189.1 at 2^24, 211.9 at 2^23).
// (src[i], dst[i]) -> pair i
__global__ void k_interleave(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint2* __restrict__ out,
                             uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = make_uint2(a[i], b[i]);
}

// Host input moves through two staging slots of at most 2^25 pairs (256 MB each side): a slice's
// copy overlaps the ingest of the previous slice, and larger slices carry the sketch update's fixed
// per-launch cost (every touched vertex's rows merged once per launch) less often.
uint64_t staging_limit(const gs_graph* g) { return std::min<uint64_t>(g->max_batch_edges, 1ull << 25); }

}  // namespace

gs_status gs_ensure_pair_staging(gs_graph* g, uint64_t want) {
  // the ring is sized for the largest host slice asked for so far (at least 2^20 pairs, a power of
  // two, at most the limit); small graphs fed small batches keep a small ring
  uint64_t target = 1ull << 20;
  while (target < want && target < staging_limit(g)) target <<= 1;
  target = std::min(target, staging_limit(g));
  if (g->d_pairs && g->pairs_cap >= target) return GS_OK;
  if (g->d_pairs) {
    // growing: every copy into and every reader of the old slots must be done
    GS_CUDA_TRY(cudaStreamSynchronize(g->copy_stream));
    for (int i = 0; i < 2; i++) GS_CUDA_TRY(cudaEventSynchronize(g->ev_done[i]));
    GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
    cudaFree(g->d_pairs);
    cudaFreeHost(g->h_pin);
    cudaFree(g->d_file_pairs);
    g->d_pairs = nullptr;
    g->h_pin = nullptr;
    g->d_file_pairs = nullptr;
    g->pairs_cap = 0;
  }
  GS_CUDA_TRY(cudaMalloc(&g->d_pairs, 2 * target * 2 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMallocHost(&g->h_pin, 2 * target * 2 * sizeof(uint32_t)));
  if (!g->copy_stream) {
    GS_CUDA_TRY(cudaStreamCreateWithFlags(&g->copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; i++) {
      GS_CUDA_TRY(cudaEventCreateWithFlags(&g->ev_copy[i], cudaEventDisableTiming));
      GS_CUDA_TRY(cudaEventCreateWithFlags(&g->ev_done[i], cudaEventDisableTiming));
    }
  }
  g->pairs_cap = target;
  return GS_OK;
}

extern "C" {

gs_status gs_graph_create(const gs_graph_config* cfg, gs_graph** out) {
  if (!cfg || !out) { gs_set_error("gs_graph_create: null argument"); return GS_ERR_BAD_ARG; }
  *out = nullptr;
  if (cfg->num_vertices < 2 || cfg->num_levels < 1 ||
      (uint64_t)cfg->num_vertices * cfg->num_levels >= (1ull << 32) - 1) {
    gs_set_error("gs_graph_create: need num_vertices >= 2, num_levels >= 1 and levels*V < 2^32");
    return GS_ERR_BAD_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    gs_set_error("no CUDA device");
    return GS_ERR_NO_DEVICE;
  }
  int dev = cfg->device;
  if (dev < 0) cudaGetDevice(&dev);
  if (dev >= ndev) { gs_set_error("device ordinal out of range"); return GS_ERR_BAD_ARG; }
  DeviceGuard guard(dev);
  if (!guard.ok) { gs_set_error("cannot select CUDA device"); return GS_ERR_NO_DEVICE; }

  std::unique_ptr<gs_graph, void (*)(gs_graph*)> g(new gs_graph(), gs_free_graph);
  g->V = cfg->num_vertices;
  g->num_levels = cfg->num_levels;
  g->num_subgraphs = cfg->num_subgraphs ? cfg->num_subgraphs : cfg->num_levels;
  if (g->num_subgraphs < 1 || g->num_subgraphs > 64) { gs_set_error("num_subgraphs must be in [1, 64]"); return GS_ERR_BAD_ARG; }
  g->seed = cfg->seed;
  g->sketches_factor = cfg->sketches_factor > 0 ? cfg->sketches_factor : 1.0;
  g->batch_factor = cfg->batch_factor > 0 ? cfg->batch_factor : 1.0;
  g->device = dev;
  g->max_batch_edges = cfg->max_batch_edges ? cfg->max_batch_edges : (1ull << 27);
  if (g->max_batch_edges > (1ull << 30)) g->max_batch_edges = 1ull << 30;
  g->store_first = g->store_initial = g->num_levels;
  g->geom = gs_make_geom(g->V, g->sketches_factor);
  if (g->geom.num_columns > 64) { gs_set_error("more than 64 sketch columns are not supported"); return GS_ERR_BAD_ARG; }
  cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, dev);
  g->tune = gs_tune_for(g->geom, g->num_sms);
  g->sample_cursor.assign(g->num_levels, 0);

  const uint32_t V = g->V, nb = g->geom.num_buckets, bkt = g->geom.bkt_per_col, C = g->geom.num_columns;
  GS_CUDA_TRY(cudaStreamCreateWithFlags(&g->own_stream, cudaStreamNonBlocking));
  g->stream = g->own_stream;
  GS_CUDA_TRY(cudaEventCreateWithFlags(&g->ev_order, cudaEventDisableTiming));
  const size_t sk_bytes = (size_t)g->num_levels * V * nb * sizeof(GsBucket);
  GS_CUDA_TRY(cudaMalloc(&g->d_sk, sk_bytes));
  GS_CUDA_TRY(cudaMemsetAsync(g->d_sk, 0, sk_bytes, g->stream));
  std::vector<uint64_t> colmix(C + 1);
  for (uint32_t c = 0; c < C; c++) colmix[c] = gs_seed_mix(g->seed + 5ull * c);  // column_seed (sketch.h:303)
  colmix[C] = gs_seed_mix(g->seed);                                                 // checksum_seed (sketch.h:304)
  GS_CUDA_TRY(cudaMalloc(&g->d_colmix, (C + 1) * sizeof(uint64_t)));
  GS_CUDA_TRY(cudaMemcpy(g->d_colmix, colmix.data(), (C + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice));
  GS_CUDA_TRY(cudaMalloc(&g->d_status, 32 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMemsetAsync(g->d_status, 0, 32 * sizeof(uint32_t), g->stream));
  GS_CUDA_TRY(cudaMallocHost(&g->h_status, 32 * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_parent, (size_t)V * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_size, (size_t)V * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_res, (size_t)V * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_samp, (size_t)V * sizeof(uint64_t)));
  GS_CUDA_TRY(cudaMalloc(&g->d_acc, (size_t)V * (bkt + 1) * sizeof(GsBucket)));
  GS_CUDA_TRY(cudaMalloc(&g->d_forest, (size_t)2 * V * sizeof(uint32_t)));
  GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  *out = g.release();
  return GS_OK;
}

gs_status gs_graph_destroy(gs_graph* g) {
  if (!g) return GS_OK;
  DeviceGuard guard(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  gs_free_graph(g);
  return GS_OK;
}

gs_status gs_graph_geometry(const gs_graph* g, gs_geometry* out) {
  if (!g || !out) { gs_set_error("null argument"); return GS_ERR_BAD_ARG; }
  out->num_vertices = g->V;
  out->num_samples = g->geom.num_samples;
  out->cols_per_sample = 1;
  out->num_columns = g->geom.num_columns;
  out->bkt_per_col = g->geom.bkt_per_col;
  out->num_buckets = g->geom.num_buckets;
  out->bytes_per_vertex = (uint64_t)g->geom.num_buckets * sizeof(GsBucket);
  return GS_OK;
}

gs_status gs_clear(gs_graph* g) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  const size_t bytes = (size_t)g->num_levels * g->V * g->geom.num_buckets * sizeof(GsBucket);
  GS_CUDA_TRY(cudaMemsetAsync(g->d_sk, 0, bytes, g->stream));
  g->labels_valid = false;
  g->changes++;
  std::fill(g->sample_cursor.begin(), g->sample_cursor.end(), 0u);
  g->store_first = g->store_initial;
  g->changes_at_clear = g->changes;
  g->sketches_symmetric = true;
  GS_TRY(gs_store_clear(g, g->stream));
  return gs_eager_reset_empty(g, g->stream);
}

gs_status gs_graph_set_stream(gs_graph* g, void* stream) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  g->stream = stream ? static_cast<cudaStream_t>(stream) : g->own_stream;
  return GS_OK;
}

uint64_t gs_desired_updates_per_batch(const gs_graph* g) {
  if (!g) return 0;
  const uint64_t n = (uint64_t)g->geom.num_buckets * sizeof(GsBucket) / sizeof(uint32_t);
  return (uint64_t)(n * g->batch_factor);
}

}  // extern "C"

namespace {

// Host input moves through the staging slots: slice k is copied on the copy stream into device slot
// k % 2 (from the caller's memory when it is page-locked, else through the pinned ring) while the
// ingest of slice k - 1 runs.  With `wait_copies`, the call returns once every copy has landed (the
// caller may reuse its buffer); without, it returns at once for page-locked input, whose buffer then
// stays in use until the handle's work is done, and every wait on a slot's earlier slice happens on
// the device, so copies of this call can run ahead of queries queued before it.
gs_status ingest_host_pairs(gs_graph* g, const uint32_t* pairs, uint64_t n, cudaStream_t s, bool wait_copies) {
  GS_TRY(gs_ensure_pair_staging(g, n));
  cudaPointerAttributes attr{};
  const bool pinned = cudaPointerGetAttributes(&attr, pairs) == cudaSuccess && attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  const uint64_t cap = g->pairs_cap;
  uint32_t* hp = static_cast<uint32_t*>(g->h_pin);
  for (uint64_t done = 0, k = 0; done < n; k++) {
    const uint64_t m = std::min(cap, n - done);
    const int slot = (int)(k & 1);
    uint32_t* dslot = g->d_pairs + (size_t)slot * cap * 2;
    const uint32_t* src = pairs + 2 * done;
    if (!pinned) {
      // the pinned slot is free once its previous copy has landed; the device slot once the ingest that
      // read it has finished
      GS_CUDA_TRY(cudaEventSynchronize(wait_copies ? g->ev_done[slot] : g->ev_copy[slot]));
      std::memcpy(hp + (size_t)slot * cap * 2, src, (size_t)m * 2 * sizeof(uint32_t));
      src = hp + (size_t)slot * cap * 2;
    } else if (wait_copies) {
      GS_CUDA_TRY(cudaEventSynchronize(g->ev_done[slot]));
    }
    GS_CUDA_TRY(cudaStreamWaitEvent(g->copy_stream, g->ev_done[slot], 0));
    GS_CUDA_TRY(cudaMemcpyAsync(dslot, src, (size_t)m * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                g->copy_stream));
    GS_CUDA_TRY(cudaEventRecord(g->ev_copy[slot], g->copy_stream));
    GS_CUDA_TRY(cudaStreamWaitEvent(s, g->ev_copy[slot], 0));
    GS_TRY(gs_ingest_device_pairs(g, dslot, m, -1, s));
    GS_CUDA_TRY(cudaEventRecord(g->ev_done[slot], s));
    done += m;
  }
  // the caller's buffer may be reused once every copy has landed
  if (wait_copies) GS_CUDA_TRY(cudaStreamSynchronize(g->copy_stream));
  return order_after(g, s);
}

constexpr uint64_t al16(uint64_t x) { return (x + 15) & ~15ull; }

// Host per-vertex batches move through the same staging slots as host pairs, so a call allocates
// nothing: the batches are cut into chunks that fit one slot (a batch longer than the room left is
// split; XOR makes the pieces equivalent to the whole), each chunk's headers and destinations are
// gathered into the slot's page-locked half - starts rebased to the gathered destinations - copied to
// the device half and ingested while the next chunk is gathered.
gs_status ingest_host_batches(gs_graph* g, uint32_t level, const uint32_t* srcs, const uint64_t* starts,
                              const uint64_t* sizes, uint32_t nbat, const uint32_t* dsts, cudaStream_t s) {
  uint64_t ndst = 0;
  for (uint32_t b = 0; b < nbat; b++) ndst += sizes[b];
  GS_TRY(gs_ensure_pair_staging(g, ndst / 2 + 3 * (uint64_t)nbat));
  const uint64_t slot_bytes = g->pairs_cap * 2 * sizeof(uint32_t);
  // a slot: batch headers (srcs u32, starts u64, sizes u64) in its first quarter, destinations after
  const uint64_t hb = std::max<uint64_t>(1, (slot_bytes / 4) / 24);
  const uint64_t off_starts = al16(hb * 4), off_sizes = off_starts + al16(hb * 8);
  const uint64_t off_dsts = al16(off_sizes + hb * 8);
  const uint64_t dcap = (slot_bytes - off_dsts) / sizeof(uint32_t);
  uint8_t* hp = static_cast<uint8_t*>(g->h_pin);
  uint8_t* dp = reinterpret_cast<uint8_t*>(g->d_pairs);
  uint32_t b = 0;
  uint64_t in_batch = 0;  // destinations of batch b already shipped
  for (int k = 0; b < nbat; k++) {
    const int slot = k & 1;
    GS_CUDA_TRY(cudaEventSynchronize(g->ev_done[slot]));   // the slot's previous chunk was ingested
    uint8_t* h = hp + slot * slot_bytes;
    uint32_t* hs = reinterpret_cast<uint32_t*>(h);
    uint64_t* hst = reinterpret_cast<uint64_t*>(h + off_starts);
    uint64_t* hsz = reinterpret_cast<uint64_t*>(h + off_sizes);
    uint32_t* hd = reinterpret_cast<uint32_t*>(h + off_dsts);
    uint64_t nb = 0, nd = 0;
    while (b < nbat && nb < hb && nd < dcap) {
      const uint64_t take = std::min(sizes[b] - in_batch, dcap - nd);
      hs[nb] = srcs[b];
      hst[nb] = nd;
      hsz[nb] = take;
      std::memcpy(hd + nd, dsts + starts[b] + in_batch, take * sizeof(uint32_t));
      nb++;
      nd += take;
      in_batch += take;
      if (in_batch == sizes[b]) { b++; in_batch = 0; }
    }
    uint8_t* d = dp + slot * slot_bytes;
    GS_CUDA_TRY(cudaMemcpyAsync(d, h, off_sizes + nb * 8, cudaMemcpyHostToDevice, s));
    if (nd) GS_CUDA_TRY(cudaMemcpyAsync(d + off_dsts, hd, nd * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    GS_TRY(gs_ingest_device_batches(g, level, reinterpret_cast<const uint32_t*>(d),
                                    reinterpret_cast<const uint64_t*>(d + off_starts),
                                    reinterpret_cast<const uint64_t*>(d + off_sizes), (uint32_t)nb,
                                    reinterpret_cast<const uint32_t*>(d + off_dsts), s, std::max<uint64_t>(nd, 1)));
    GS_CUDA_TRY(cudaEventRecord(g->ev_done[slot], s));
  }
  return order_after(g, s);
}

}  // namespace

extern "C" {

gs_status gs_prepare_host_input(gs_graph* g, uint64_t records) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  GS_TRY(gs_ensure_pair_staging(g, records));
  if (!g->d_file_pairs) {
    const uint64_t per = g->pairs_cap * 2 * sizeof(uint32_t) / 9;  // stream-file records per slice
    GS_CUDA_TRY(cudaMalloc(&g->d_file_pairs, per * sizeof(uint2)));
  }
  return GS_OK;
}

gs_status gs_ingest_pairs(gs_graph* g, const uint32_t* pairs, uint64_t n, int on_device, void* stream) {
  if (!g || (n && !pairs)) { gs_set_error("gs_ingest_pairs: null argument"); return GS_ERR_BAD_ARG; }
  if (n == 0) return GS_OK;
  GS_GUARD(g);
  cudaStream_t s = pick_stream(g, stream);
  g->labels_valid = false;
  g->changes++;
  if (on_device) {
    GS_TRY(gs_ingest_device_pairs(g, pairs, n, -1, s));
    return order_after(g, s);
  }
  return ingest_host_pairs(g, pairs, n, s, true);
}

gs_status gs_ingest_pairs_async(gs_graph* g, const uint32_t* pairs, uint64_t n, int on_device, void* stream) {
  if (!g || (n && !pairs)) { gs_set_error("gs_ingest_pairs_async: null argument"); return GS_ERR_BAD_ARG; }
  if (n == 0) return GS_OK;
  GS_GUARD(g);
  cudaStream_t s = pick_stream(g, stream);
  g->labels_valid = false;
  g->changes++;
  if (on_device) {
    GS_TRY(gs_ingest_device_pairs(g, pairs, n, -1, s));
    return order_after(g, s);
  }
  return ingest_host_pairs(g, pairs, n, s, false);
}

gs_status gs_ingest_edges(gs_graph* g, const uint32_t* src, const uint32_t* dst, uint64_t n, int on_device,
                          void* stream) {
  if (!g || (n && (!src || !dst))) { gs_set_error("gs_ingest_edges: null argument"); return GS_ERR_BAD_ARG; }
  if (n == 0) return GS_OK;
  GS_GUARD(g);
  if (!on_device) {
    std::vector<uint32_t> host(2 * n);
    for (uint64_t i = 0; i < n; i++) { host[2 * i] = src[i]; host[2 * i + 1] = dst[i]; }
    return gs_ingest_pairs(g, host.data(), n, 0, stream);
  }
  // device arrays: interleaved on the device into the staging slots, one slice at a time
  cudaStream_t s = pick_stream(g, stream);
  g->labels_valid = false;
  g->changes++;
  GS_TRY(gs_ensure_pair_staging(g, n));
  const uint64_t cap = g->pairs_cap;
  for (uint64_t done = 0, k = 0; done < n; k++) {
    const uint64_t m = std::min(cap, n - done);
    const int slot = (int)(k & 1);
    uint32_t* dslot = g->d_pairs + (size_t)slot * cap * 2;
    // the slot's previous slice must be consumed before it is overwritten
    GS_CUDA_TRY(cudaStreamWaitEvent(s, g->ev_done[slot], 0));
    const int grid = (int)std::min<uint64_t>((m + 255) / 256, (uint64_t)g->num_sms * 8);
    k_interleave<<<grid, 256, 0, s>>>(src + done, dst + done, reinterpret_cast<uint2*>(dslot), m);
    GS_CUDA_TRY(cudaGetLastError());
    GS_TRY(gs_ingest_device_pairs(g, dslot, m, -1, s));
    GS_CUDA_TRY(cudaEventRecord(g->ev_done[slot], s));
    done += m;
  }
  return order_after(g, s);
}

gs_status gs_ingest_vertex_batches(gs_graph* g, uint32_t level, const uint32_t* srcs, const uint64_t* starts,
                                   const uint64_t* sizes, uint32_t nbat, const uint32_t* dsts, uint64_t ndst,
                                   int on_device, void* stream) {
  if (!g || (nbat && (!srcs || !starts || !sizes)) || (ndst && !dsts)) {
    gs_set_error("gs_ingest_vertex_batches: null argument");
    return GS_ERR_BAD_ARG;
  }
  if (level >= g->num_levels) { gs_set_error("level out of range"); return GS_ERR_BAD_ARG; }
  if (nbat == 0) return GS_OK;
  GS_GUARD(g);
  cudaStream_t s = pick_stream(g, stream);
  g->labels_valid = false;
  g->changes++;
  g->sketches_symmetric = false;  // one-sided updates: the XOR of all vertex sketches is no longer zero
  if (on_device) {
    GS_TRY(gs_ingest_device_batches(g, level, srcs, starts, sizes, nbat, dsts, s));
    return order_after(g, s);
  }
  for (uint32_t b = 0; b < nbat; b++) {
    if (starts[b] > ndst || sizes[b] > ndst - starts[b]) {
      gs_set_error("gs_ingest_vertex_batches: batch " + std::to_string(b) + " exceeds the dst array");
      return GS_ERR_BAD_ARG;
    }
  }
  return ingest_host_batches(g, level, srcs, starts, sizes, nbat, dsts, s);
}

gs_status gs_synchronize(gs_graph* g) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  if (g->copy_stream) GS_CUDA_TRY(cudaStreamSynchronize(g->copy_stream));
  return check_status(g, g->stream);
}

gs_status gs_connected_components(gs_graph* g, uint32_t level, uint32_t* labels, uint32_t* num_cc, uint32_t* rounds) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  if (level >= g->num_levels) { gs_set_error("level out of range"); return GS_ERR_BAD_ARG; }
  if (g->query_pending) { gs_set_error("a queued query is pending: collect it with gs_query_wait first"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  cudaStream_t s = g->stream;
  GS_TRY(check_status(g, s));
  bool cached = false;
  if (level == 0) GS_TRY(gs_eager_state(g, s, &cached));
  if (cached) {
    GS_TRY(gs_eager_answer(g, s));   // CCSketchAlg::connected_components with shared_dsu_valid
  } else {
    GS_TRY(gs_boruvka(g, level, 0, s));
    g->last_answer_eager = false;
    if (level == 0) GS_TRY(gs_eager_rebuild(g, s));
  }
  if (rounds) *rounds = g->last_rounds;
  if (labels || num_cc) {
    std::vector<uint32_t> tmp;
    uint32_t* dst = labels;
    if (!dst) { tmp.resize(g->V); dst = tmp.data(); }
    GS_CUDA_TRY(cudaMemcpyAsync(dst, g->d_parent, (size_t)g->V * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GS_CUDA_TRY(cudaStreamSynchronize(s));
    if (num_cc) {
      uint32_t c = 0;
      for (uint32_t v = 0; v < g->V; v++) c += dst[v] == v;
      *num_cc = c;
    }
  }
  return GS_OK;
}

gs_status gs_connected_components_async(gs_graph* g, uint32_t level) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  if (level >= g->num_levels) { gs_set_error("level out of range"); return GS_ERR_BAD_ARG; }
  if (g->query_pending) { gs_set_error("a queued query is pending: collect it with gs_query_wait first"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  cudaStream_t s = g->stream;
  if (!g->h_qlabels) {
    GS_CUDA_TRY(cudaMallocHost(&g->h_qstatus, 32 * sizeof(uint32_t)));
    GS_CUDA_TRY(cudaMallocHost(&g->h_qlabels, (size_t)g->V * sizeof(uint32_t)));
    GS_CUDA_TRY(cudaEventCreateWithFlags(&g->ev_query, cudaEventDisableTiming));
  }
  g->query_level = level;
  g->query_changes = g->changes;
  g->query_done = false;
  g->query_status = GS_OK;
  if (level == 0 && g->eager_on) {
    // the eager DSU answers at once (it synchronizes anyway); gs_query_wait hands the answer out
    uint32_t ncc = 0, rounds = 0;
    g->query_status = gs_connected_components(g, 0, g->h_qlabels, &ncc, &rounds);
    g->h_qstatus[0] = ncc;
    g->h_qstatus[1] = rounds;
    g->query_done = true;
    g->query_pending = true;
    return GS_OK;
  }
  GS_TRY(gs_boruvka_enqueue(g, level, 0, s, g->h_qstatus));
  GS_CUDA_TRY(cudaMemcpyAsync(g->h_qlabels, g->d_parent, (size_t)g->V * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GS_CUDA_TRY(cudaEventRecord(g->ev_query, s));
  g->query_pending = true;
  return GS_OK;
}

gs_status gs_query_wait(gs_graph* g, uint32_t* labels, uint32_t* num_cc, uint32_t* rounds) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  if (!g->query_pending) { gs_set_error("gs_query_wait: no query is queued"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  g->query_pending = false;
  const uint32_t V = g->V;
  if (g->query_done) {
    if (g->query_status != GS_OK) return g->query_status;
    if (labels) std::memcpy(labels, g->h_qlabels, (size_t)V * sizeof(uint32_t));
    if (num_cc) *num_cc = g->h_qstatus[0];
    if (rounds) *rounds = g->h_qstatus[1];
    return GS_OK;
  }
  GS_CUDA_TRY(cudaEventSynchronize(g->ev_query));
  const uint32_t* st = g->h_qstatus;
  if (st[16] & GS_DEV_ERR_VERTEX_RANGE) {
    // as gs_connected_components, which reports records skipped by earlier ingest calls first
    gs_set_error("an edge record named a vertex id >= num_vertices; those records were skipped");
    g->acc_dirty = true;
    return GS_ERR_BAD_ARG;
  }
  if (st[16]) {
    gs_set_error("device consistency check failed (bits " + std::to_string(st[16]) + ")");
    g->acc_dirty = true;
    return GS_ERR_INTERNAL;
  }
  GS_TRY(gs_boruvka_finish(g, g->query_level, st));
  g->last_answer_eager = false;
  // the partition stays valid for point queries only while no later call has changed the sketches
  g->labels_valid = g->changes == g->query_changes;
  if (g->query_level == 0 && g->eager_on) GS_TRY(gs_eager_rebuild(g, g->stream));
  if (rounds) *rounds = g->last_rounds;
  if (labels) std::memcpy(labels, g->h_qlabels, (size_t)V * sizeof(uint32_t));
  if (num_cc) {
    uint32_t c = 0;
    for (uint32_t v = 0; v < V; v++) c += g->h_qlabels[v] == v;
    *num_cc = c;
  }
  return GS_OK;
}

gs_status gs_point_query(gs_graph* g, uint32_t a, uint32_t b, int* connected) {
  if (!g || !connected || a >= g->V || b >= g->V) { gs_set_error("gs_point_query: bad arguments"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  if (!g->labels_valid || g->labels_level != 0) GS_TRY(gs_connected_components(g, 0, nullptr, nullptr, nullptr));
  uint32_t ra = 0, rb = 0;
  GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  GS_CUDA_TRY(cudaMemcpy(&ra, g->d_parent + a, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  GS_CUDA_TRY(cudaMemcpy(&rb, g->d_parent + b, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  *connected = ra == rb;
  return GS_OK;
}

gs_status gs_spanning_forest(gs_graph* g, uint32_t level, uint32_t* edges, uint64_t* num_edges) {
  if (!g || !edges || !num_edges) { gs_set_error("gs_spanning_forest: null argument"); return GS_ERR_BAD_ARG; }
  GS_TRY(gs_connected_components(g, level, nullptr, nullptr, nullptr));
  GS_GUARD(g);
  if (g->last_answer_eager) GS_TRY(gs_eager_forest(g, g->stream));  // the eager forest, as the reference returns
  *num_edges = g->last_forest_edges;
  GS_CUDA_TRY(cudaMemcpy(edges, g->d_forest, (size_t)2 * g->last_forest_edges * sizeof(uint32_t),
                         cudaMemcpyDeviceToHost));
  return GS_OK;
}

gs_status gs_disjoint_spanning_forests(gs_graph* g, uint32_t level, uint32_t k, uint32_t* edges, uint64_t* sizes) {
  if (!g || !edges || !sizes || k == 0) { gs_set_error("gs_disjoint_spanning_forests: bad arguments"); return GS_ERR_BAD_ARG; }
  if (g->query_pending) { gs_set_error("a queued query is pending: collect it with gs_query_wait first"); return GS_ERR_BAD_ARG; }
  if (level >= g->num_levels) { gs_set_error("level out of range"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  cudaStream_t s = g->stream;
  GS_TRY(check_status(g, s));
  const uint32_t V = g->V;
  const size_t stride = 2 * (size_t)(V - 1);
  uint32_t* d_all = nullptr;
  GS_CUDA_TRY(cudaMalloc(&d_all, std::max<size_t>(1, k * stride) * sizeof(uint32_t)));
  uint64_t total = 0;
  gs_status st = GS_OK;
  uint32_t done = 0;
  for (uint32_t j = 0; j < k; j++) {
    // a min-cut graph samples round 0 at the column its stored sample index reached; a
    // connected-components graph resets it before every query (CCSketchAlg::connected_components)
    const uint32_t col0 = (g->num_levels > 1 || g->num_subgraphs > 1) ? g->sample_cursor[level]++ : 0;
    st = gs_boruvka(g, level, col0, s);
    if (st != GS_OK) break;
    const uint32_t ne = g->last_forest_edges;
    sizes[j] = ne;
    cudaMemcpyAsync(d_all + total * 2, g->d_forest, (size_t)2 * ne * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(edges + j * stride, g->d_forest, (size_t)2 * ne * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    // filter_sf_edges: XOR the forest out of both endpoint sketches of this level
    st = gs_ingest_device_pairs(g, d_all + total * 2, ne, (int)level, s);
    total += ne;
    done++;
    if (st != GS_OK) break;
  }
  // re-insert every forest found so far (src/mc_sketch_alg.cpp:904-907)
  gs_status st2 = total ? gs_ingest_device_pairs(g, d_all, total, (int)level, s) : GS_OK;
  cudaStreamSynchronize(s);
  cudaFree(d_all);
  for (uint32_t j = done; j < k; j++) sizes[j] = 0;
  g->labels_valid = false;
  g->changes++;
  gs_eager_invalidate(g, s);  // the parent array now holds the last forest's partition
  if (st != GS_OK) return st;
  if (st2 != GS_OK) return st2;
  GS_CUDA_TRY(cudaGetLastError());
  return check_status(g, s);
}

gs_status gs_min_cut(gs_graph* g, uint32_t k, uint64_t* value, uint32_t* level_found, uint64_t* cut_at_level,
                     uint8_t* side) {
  if (!g || !value || k == 0) { gs_set_error("gs_min_cut: bad arguments"); return GS_ERR_BAD_ARG; }
  const uint32_t V = g->V;
  std::vector<uint32_t> edges((size_t)k * 2 * (V - 1));
  std::vector<uint64_t> sizes(k);
  // the levels sketched now (all configured levels unless the exact tier is adaptive)
  const uint32_t sketched = g->store_first;
  for (uint32_t lvl = 0; lvl < sketched; lvl++) {
    GS_TRY(gs_disjoint_spanning_forests(g, lvl, k, edges.data(), sizes.data()));
    std::vector<uint32_t> cert;
    for (uint32_t f = 0; f < k; f++)
      cert.insert(cert.end(), edges.begin() + (size_t)f * 2 * (V - 1),
                  edges.begin() + (size_t)f * 2 * (V - 1) + 2 * sizes[f]);
    const uint64_t cut = gs_exact_min_cut_host(V, cert.data(), cert.size() / 2, side);
    if (cut < k || (lvl + 1 == sketched && !gs_store_active(g))) {
      *value = cut << lvl;
      if (level_found) *level_found = lvl;
      if (cut_at_level) *cut_at_level = cut;
      return GS_OK;
    }
  }
  // no sketched level certified a cut below k: the first unsketched level answers whatever its
  // value, with the exact minimum cut of all its edges from the exact tier (tools/min_cut.cu:221-247;
  // get_adjlist_spanning_forests returns the store's whole edge list, src/mc_gpu_sketch_alg.cpp:207-209)
  const uint32_t lvl = sketched;
  {
    GS_GUARD(g);
    GS_TRY(check_status(g, g->stream));
    std::vector<uint32_t> exact;
    GS_TRY(gs_store_edges(g, lvl, &exact, g->stream));
    const uint64_t cut = gs_exact_min_cut_host(V, exact.data(), exact.size() / 2, side);
    *value = cut << lvl;
    if (level_found) *level_found = lvl;
    if (cut_at_level) *cut_at_level = cut;
  }
  return GS_OK;
}

gs_status gs_graph_set_edge_store(gs_graph* g, uint32_t initial_sketch_levels, uint64_t store_bytes) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  if (initial_sketch_levels > g->num_levels || g->num_subgraphs <= 1) {
    gs_set_error("gs_graph_set_edge_store: a min-cut graph (num_subgraphs > 1) and initial_sketch_levels <= num_levels");
    return GS_ERR_BAD_ARG;
  }
  if (g->changes != g->changes_at_clear) {
    gs_set_error("gs_graph_set_edge_store: set the exact tier before the first ingest (or right after gs_clear)");
    return GS_ERR_BAD_ARG;
  }
  GS_GUARD(g);
  const uint64_t level_bytes = (uint64_t)g->V * g->geom.num_buckets * sizeof(GsBucket);
  g->store_initial = g->store_first = initial_sketch_levels;
  g->store_adaptive = true;
  g->store_budget = std::max<uint64_t>(1, (store_bytes ? store_bytes : level_bytes) / 16);
  if (g->d_store) {   // sized for the default budget: the next tagged ingest sizes it again
    cudaFree(g->d_store);
    g->d_store = nullptr;
  }
  return GS_OK;
}

gs_status gs_graph_sketched_levels(const gs_graph* g, uint32_t* levels, uint64_t* contractions) {
  if (!g || !levels) { gs_set_error("null argument"); return GS_ERR_BAD_ARG; }
  *levels = g->store_first;
  if (contractions) *contractions = g->store_contractions;
  return GS_OK;
}

gs_status gs_edge_store_edges(gs_graph* g, uint32_t min_tag, uint32_t* edges, uint64_t capacity, uint64_t* num_edges) {
  if (!g || !num_edges || (capacity && !edges)) { gs_set_error("gs_edge_store_edges: bad arguments"); return GS_ERR_BAD_ARG; }
  GS_GUARD(g);
  GS_TRY(check_status(g, g->stream));
  std::vector<uint32_t> exact;
  GS_TRY(gs_store_edges(g, min_tag, &exact, g->stream));
  std::vector<uint64_t> ids(exact.size() / 2);
  for (size_t i = 0; i < ids.size(); i++) ids[i] = ((uint64_t)exact[2 * i] << 32) | exact[2 * i + 1];
  std::sort(ids.begin(), ids.end());
  *num_edges = ids.size();
  for (size_t i = 0; i < ids.size() && i < capacity; i++) {
    edges[2 * i] = (uint32_t)(ids[i] >> 32);
    edges[2 * i + 1] = (uint32_t)ids[i];
  }
  return GS_OK;
}

gs_status gs_download_sketches(gs_graph* g, uint32_t level, uint32_t first, uint32_t count, void* host_out) {
  if (!g || !host_out || level >= g->num_levels || (uint64_t)first + count > g->V) {
    gs_set_error("gs_download_sketches: bad arguments");
    return GS_ERR_BAD_ARG;
  }
  GS_GUARD(g);
  GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  const size_t nb = g->geom.num_buckets;
  GS_CUDA_TRY(cudaMemcpy(host_out, g->d_sk + ((size_t)level * g->V + first) * nb, (size_t)count * nb * sizeof(GsBucket),
                         cudaMemcpyDeviceToHost));
  return GS_OK;
}

gs_status gs_upload_sketches(gs_graph* g, uint32_t level, uint32_t first, uint32_t count, const void* host_in) {
  if (!g || !host_in || level >= g->num_levels || (uint64_t)first + count > g->V) {
    gs_set_error("gs_upload_sketches: bad arguments");
    return GS_ERR_BAD_ARG;
  }
  GS_GUARD(g);
  GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  const size_t nb = g->geom.num_buckets;
  GS_CUDA_TRY(cudaMemcpy(g->d_sk + ((size_t)level * g->V + first) * nb, host_in, (size_t)count * nb * sizeof(GsBucket),
                         cudaMemcpyHostToDevice));
  g->sketches_symmetric = false;  // arbitrary bytes: nothing is known about their XOR
  g->labels_valid = false;
  g->changes++;
  return gs_eager_invalidate(g, g->stream);
}

gs_status gs_write_binary(gs_graph* g, const char* path) {
  if (!g || !path) { gs_set_error("gs_write_binary: null argument"); return GS_ERR_BAD_ARG; }
  FILE* f = std::fopen(path, "wb");
  if (!f) { gs_set_error(std::string("cannot open ") + path); return GS_ERR_IO; }
  const uint64_t seed = g->seed;
  const uint32_t V = g->V;
  const double factor = g->sketches_factor;
  bool ok = std::fwrite(&seed, 8, 1, f) == 1 && std::fwrite(&V, 4, 1, f) == 1 && std::fwrite(&factor, 8, 1, f) == 1;
  const size_t nb = g->geom.num_buckets;
  const uint32_t step = (uint32_t)std::max<size_t>(1, (64u << 20) / (nb * sizeof(GsBucket)));
  std::vector<GsBucket> buf((size_t)step * nb);
  for (uint32_t v = 0; ok && v < V; v += step) {
    const uint32_t c = std::min(step, V - v);
    gs_status st = gs_download_sketches(g, 0, v, c, buf.data());
    if (st != GS_OK) { std::fclose(f); return st; }
    ok = std::fwrite(buf.data(), sizeof(GsBucket), (size_t)c * nb, f) == (size_t)c * nb;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { gs_set_error(std::string("write failed: ") + path); return GS_ERR_IO; }
  return GS_OK;
}

gs_status gs_read_binary(const char* path, int32_t device, gs_graph** out) {
  if (!path || !out) { gs_set_error("gs_read_binary: null argument"); return GS_ERR_BAD_ARG; }
  FILE* f = std::fopen(path, "rb");
  if (!f) { gs_set_error(std::string("cannot open ") + path); return GS_ERR_IO; }
  uint64_t seed = 0;
  uint32_t V = 0;
  double factor = 1;
  if (std::fread(&seed, 8, 1, f) != 1 || std::fread(&V, 4, 1, f) != 1 || std::fread(&factor, 8, 1, f) != 1) {
    std::fclose(f);
    gs_set_error("truncated header");
    return GS_ERR_IO;
  }
  gs_graph_config cfg{};
  cfg.num_vertices = V;
  cfg.num_levels = 1;
  cfg.seed = seed;
  cfg.sketches_factor = factor;
  cfg.batch_factor = 1;
  cfg.device = device;
  gs_graph* g = nullptr;
  gs_status st = gs_graph_create(&cfg, &g);
  if (st != GS_OK) { std::fclose(f); return st; }
  const size_t nb = g->geom.num_buckets;
  const uint32_t step = (uint32_t)std::max<size_t>(1, (64u << 20) / (nb * sizeof(GsBucket)));
  std::vector<GsBucket> buf((size_t)step * nb);
  for (uint32_t v = 0; v < V; v += step) {
    const uint32_t c = std::min(step, V - v);
    if (std::fread(buf.data(), sizeof(GsBucket), (size_t)c * nb, f) != (size_t)c * nb) {
      std::fclose(f);
      gs_graph_destroy(g);
      gs_set_error("truncated sketch data");
      return GS_ERR_IO;
    }
    st = gs_upload_sketches(g, 0, v, c, buf.data());
    if (st != GS_OK) { std::fclose(f); gs_graph_destroy(g); return st; }
  }
  std::fclose(f);
  *out = g;
  return GS_OK;
}

gs_status gs_gen_rmat_stream(uint32_t log2_v, double a, double b, double c, double delete_frac, uint64_t seed,
                             uint64_t first, uint64_t n, uint32_t* pairs, int on_device, void* stream) {
  if ((n && !pairs) || log2_v < 1 || log2_v > 31 || a < 0 || b < 0 || c < 0 || a + b + c > 1) {
    gs_set_error("gs_gen_rmat_stream: bad arguments");
    return GS_ERR_BAD_ARG;
  }
  if (on_device) {
    GS_TRY(gs_gen_rmat_device(log2_v, a, b, c, delete_frac, seed, first, n, pairs, static_cast<cudaStream_t>(stream)));
    return GS_OK;
  }
  gs_gen_rmat_host(log2_v, a, b, c, delete_frac, seed, first, n, pairs);
  return GS_OK;
}

}  // extern "C"

// ---- eager DSU ----

extern "C" gs_status gs_set_eager_dsu(gs_graph* g, int enable) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  DeviceGuard guard(g->device);
  return gs_eager_enable(g, enable != 0, g->stream);
}

extern "C" gs_status gs_has_cached_query(gs_graph* g, int* cached) {
  if (!g || !cached) { gs_set_error("null argument"); return GS_ERR_BAD_ARG; }
  DeviceGuard guard(g->device);
  bool v = false;
  GS_TRY(gs_eager_state(g, g->stream, &v));
  *cached = v ? 1 : 0;
  return GS_OK;
}

// ---- bounded device-side waits ----

extern "C" gs_status gs_set_device_wait_limit(gs_graph* g, uint64_t nanoseconds) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  g->wait_ns = nanoseconds ? nanoseconds : kGsDefaultWaitNs;
  return GS_OK;
}

// ---- tuning ----

extern "C" gs_status gs_get_tuning(const gs_graph* g, gs_tuning* out) {
  if (!g || !out) { gs_set_error("null argument"); return GS_ERR_BAD_ARG; }
  out->chunk = g->tune.chunk;
  out->warps_per_block = g->tune.warps_per_block;
  out->reg_depth = g->tune.reg_depth;
  out->reserved = 0;
  return GS_OK;
}

extern "C" gs_status gs_set_tuning(gs_graph* g, const gs_tuning* t) {
  if (!g || !t) { gs_set_error("null argument"); return GS_ERR_BAD_ARG; }
  if (t->chunk < 32 || t->chunk > (1u << 20) || t->warps_per_block < 1 || t->warps_per_block > 16 ||
      t->reg_depth > 3) {
    gs_set_error("gs_set_tuning: chunk in [32, 2^20], warps_per_block in [1, 16], reg_depth in [0, 3]");
    return GS_ERR_BAD_ARG;
  }
  g->tune.chunk = t->chunk;
  g->tune.warps_per_block = t->warps_per_block;
  g->tune.reg_depth = t->reg_depth;
  return GS_OK;
}

// ---- profiling ----

GsProfScope::GsProfScope(gs_graph* g_, int cls_, cudaStream_t s_, uint32_t launches) : g(g_), cls(cls_), s(s_) {
  g->prof_launches[cls] += launches;
  g->launches_total += launches;
  if (!g->prof_on || g->capturing) return;
  auto& ev = g->prof_ev[cls];
  const size_t i = g->prof_used[cls];
  if (ev.size() < 2 * (i + 1)) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return;
    ev.push_back(a);
    ev.push_back(b);
  }
  if (cudaEventRecord(ev[2 * i], s) != cudaSuccess) return;
  idx = (long)i;
  g->prof_used[cls] = i + 1;
}

GsProfScope::~GsProfScope() {
  if (idx >= 0) cudaEventRecord(g->prof_ev[cls][2 * idx + 1], s);
}

extern "C" gs_status gs_profile_enable(gs_graph* g, int enable) {
  if (!g) { gs_set_error("null handle"); return GS_ERR_BAD_ARG; }
  DeviceGuard guard(g->device);
  cudaStreamSynchronize(g->stream);
  g->prof_on = enable != 0;
  for (int c = 0; c < 3; c++) { g->prof_used[c] = 0; g->prof_launches[c] = 0; }
  g->launches_total = 0;
  g->records_total = 0;
  return GS_OK;
}

extern "C" gs_status gs_profile_read(gs_graph* g, gs_profile* out) {
  if (!g || !out) { gs_set_error("null argument"); return GS_ERR_BAD_ARG; }
  DeviceGuard guard(g->device);
  GS_CUDA_TRY(cudaStreamSynchronize(g->stream));
  double ms[3] = {0, 0, 0};
  for (int c = 0; c < 3; c++) {
    for (size_t i = 0; i < g->prof_used[c]; i++) {
      float t = 0;
      GS_CUDA_TRY(cudaEventElapsedTime(&t, g->prof_ev[c][2 * i], g->prof_ev[c][2 * i + 1]));
      ms[c] += t;
    }
  }
  out->ingest_launches = g->prof_launches[GS_PROF_INGEST];
  out->ingest_ms = ms[GS_PROF_INGEST];
  out->bucket_launches = g->prof_launches[GS_PROF_BUCKET];
  out->bucket_ms = ms[GS_PROF_BUCKET];
  out->query_launches = g->prof_launches[GS_PROF_QUERY];
  out->query_ms = ms[GS_PROF_QUERY];
  out->kernel_launches = g->launches_total;
  out->records_ingested = g->records_total;
  return GS_OK;
}
