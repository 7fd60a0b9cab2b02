// gs_internal.h - the gs_graph handle and the launchers shared by the library's .cu files.
#pragma once

#include <cstdint>
#include <vector>

#include "gs_common.cuh"

// Default limit of a bounded device-side wait (the Boruvka grid barriers): about a second.
constexpr uint64_t kGsDefaultWaitNs = 1000000000ull;

// Column-constant row of one engine tenant: num_columns column constants, then the checksum constant.
constexpr uint32_t kColStride = 65;

// Geometry and arena placement of one engine tenant, as the ingest kernels read it.
struct GsIngTenant {
  uint64_t sk_off;   // bucket offset of the tenant's vertex-0 sketch in the arena
  uint32_t vbase;    // first vertex of the tenant in the engine's vertex space
  uint32_t V, C, bkt, nb, pad;
};

// One entry of the eager DSU's forest set: an edge id (0 = empty), the ingest batch that added it,
// and how often that batch toggled it.
struct GsEagerSlot {
  uint64_t key;
  uint32_t epoch;
  uint32_t count;
};

// One entry of the exact tier of deep min-cut levels (gs_store.cu): an edge id (0 = empty), its
// subgraph tag and the parity of its toggles (odd = present).
struct GsStoreSlot {
  uint64_t key;
  uint32_t tag;
  uint32_t parity;
};

// Ingest tuning knobs (picked per geometry by gs_tune_for; overridable through
// gs_set_tuning for the autotuner).
struct GsTuning {
  uint32_t chunk;            // records per work item; larger vertices are split across warps
  uint32_t warps_per_block;  // warps in an ingest block
  uint32_t reg_depth;        // bucket depths each lane keeps in registers (1..3)
};

struct gs_graph {
  // ---- configuration ----
  GsGeom geom{};
  uint32_t V = 0;
  uint32_t num_levels = 1;
  uint32_t num_subgraphs = 1;  // min-cut tag bound L
  uint64_t seed = 0;
  double sketches_factor = 1.0;
  double batch_factor = 1.0;
  int device = 0;
  int num_sms = 148;
  uint64_t max_batch_edges = 1ull << 27;
  GsTuning tune{};
  cudaStream_t stream = nullptr;      // stream every kernel of this handle is launched on
  cudaStream_t own_stream = nullptr;  // created with the handle
  cudaEvent_t ev_order = nullptr;     // orders the handle's stream after a caller-stream ingest

  // ---- resident state ----
  GsBucket* d_sk = nullptr;    // [num_levels][V][num_buckets]
  uint64_t* d_colmix = nullptr;  // [num_columns] mix(B(seed+5c)), then [num_columns] = mix(B(seed))

  // ---- engine tenants (set only on the plumbing handle of a gs_engine) ----
  const uint32_t* d_vtenant = nullptr;  // [V] tenant of each vertex of the engine's vertex space
  const GsIngTenant* d_ten = nullptr;   // tenant geometry table; d_colmix then holds kColStride per tenant
  uint32_t ten_max_cols = 0;            // most columns of any live tenant
  uint32_t ten_min_bkt = 0;             // fewest buckets per column of any live tenant

  // ---- ingest scratch ----
  uint64_t nv_cap = 0;         // virtual vertices the per-vertex arrays hold (num_levels*V)
  uint32_t* d_cnt = nullptr;   // [nv+1] records per virtual vertex, then cursors
  uint32_t* d_off = nullptr;   // [nv+1] exclusive scan of d_cnt
  uint32_t* d_choff = nullptr; // [nv+1] exclusive scan of d_nch
  uint32_t* d_tile = nullptr;  // [2*tiles] per-tile sums for the scan
  uint32_t* d_nbr = nullptr;   // [nbr_cap] neighbour of each record, grouped by virtual vertex
  uint64_t nbr_cap = 0;
  uint2* d_part = nullptr;     // [part_cap] (key, neighbour) records partitioned by key >> part_lb
  uint64_t part_cap = 0;
  uint32_t* d_bkt = nullptr;   // bucket tables of the partition: tot[H] off[H+1] cur[H] choff[H+1]
  uint32_t* d_blockhist = nullptr;  // [tiles][H] bucket counts of every pass-1 block
  uint64_t blockhist_cap = 0;
  uint32_t* d_chunkhist = nullptr;  // [chunks][2^lb] vertex counts of every pass-2 chunk
  uint64_t chunkhist_cap = 0;
  uint32_t* d_owner = nullptr;      // [work chunk] vertex owning it, for the chunks below owner_cap
  uint64_t owner_cap = 0;
  uint32_t part_buckets = 0;   // H
  uint32_t part_lb = 9;        // low key bits resolved by the second pass
  uint32_t* d_pairs = nullptr; // staging for host-resident input pairs, 2 x [pairs_cap] u32 pairs
  uint64_t pairs_cap = 0;
  void* h_pin = nullptr;       // 2 pinned staging buffers of pairs_cap pairs
  uint2* d_file_pairs = nullptr; // decoded records of one stream-file slice (gs_ingest_stream_file)
  cudaStream_t copy_stream = nullptr;               // H2D of host input slices
  cudaEvent_t ev_copy[2] = {nullptr, nullptr};      // slice copied into d_pairs[slot]
  cudaEvent_t ev_done[2] = {nullptr, nullptr};      // slice in d_pairs[slot] consumed
  uint32_t* d_status = nullptr;  // [0] error bits [1] records [2] chunks [3] modified [4] forest [5] part chunks
                                 // ... [16] ingest error bits carried across a query (32 words)
  uint32_t* h_status = nullptr;  // pinned mirror (32 words)
  uint64_t changes = 0;          // count of calls that changed the sketches
  uint64_t changes_at_clear = 0; // `changes` right after the last gs_clear (0: none since creation)

  // ---- asynchronous query (gs_connected_components_async / gs_query_wait) ----
  bool query_pending = false;
  uint32_t query_level = 0;
  uint64_t query_changes = 0;      // `changes` when the query was queued
  gs_status query_status = GS_OK;  // answer already known at submission (eager DSU, or an error)
  bool query_done = false;
  uint32_t* h_qstatus = nullptr;   // pinned, 32 words: the query's status words
  uint32_t* h_qlabels = nullptr;   // pinned, V labels
  cudaEvent_t ev_query = nullptr;  // recorded after the labels' read-back

  // ---- Boruvka scratch ----
  uint32_t* d_parent = nullptr;  // [V]
  uint32_t* d_size = nullptr;    // [V]
  uint32_t* d_res = nullptr;     // [V] sample result code
  uint64_t* d_samp = nullptr;    // [V] sampled edge id
  GsBucket* d_acc = nullptr;     // [V][bkt_per_col+1] merged column + deterministic bucket
  bool acc_dirty = true;         // d_acc may hold non-zero rows (new, or a query ended early)
  uint32_t* d_forest = nullptr;  // [2*(V-1)] forest edges of the last Boruvka run
  uint32_t last_forest_edges = 0;
  uint32_t last_rounds = 0;
  std::vector<uint32_t> sample_cursor;  // per level: round-0 column of the next k-forest
  bool labels_valid = false;     // d_parent holds the partition of the last query
  uint32_t labels_level = 0;
  uint64_t wait_ns = kGsDefaultWaitNs;  // limit of the Boruvka kernel's grid-barrier waits
  // Every update so far reached both endpoints' sketches (edge records, forests XORed out and back),
  // so on every level the XOR of all vertex sketches is zero.  One-sided vertex batches and uploaded
  // sketches clear it; gs_clear sets it again.
  bool sketches_symmetric = true;

  // ---- eager DSU (gs_eager.cu): connectivity kept current by the ingest path ----
  bool eager_on = false;
  bool last_answer_eager = false;     // the last CC answer came from the eager DSU, not Boruvka
  GsEagerSlot* d_eager_set = nullptr; // forest edge set, eager_mask + 1 slots
  uint32_t* d_eager_status = nullptr; // [0] invalid (non-zero) [1] error bits [2] scratch counter
  uint32_t* h_eager = nullptr;        // pinned mirror of the status words
  uint32_t eager_mask = 0;
  uint32_t eager_epoch = 0;
  uint64_t eager_answers = 0;

  // ---- exact tier of the deep min-cut levels (gs_store.cu) ----
  GsStoreSlot* d_store = nullptr;     // allocated at the first tagged ingest that needs it
  uint32_t* d_store_status = nullptr; // [0] live edges [1] error bits [2] slots used [3] scratch counter
  uint32_t* h_store = nullptr;        // pinned mirror
  uint32_t store_mask = 0;
  // sketched levels: records tag into levels 0..min(tag, store_first-1), edges with tag >= store_first
  // are kept exactly.  store_first starts at store_initial and grows by one per contraction while it
  // is below num_levels (gs_graph_set_edge_store); without that call it stays num_levels.
  uint32_t store_first = 1;
  uint32_t store_initial = 1;
  bool store_adaptive = false;
  uint64_t store_budget = 0;          // live edges that trigger a contraction
  uint64_t store_contractions = 0;
  uint2* d_store_list = nullptr;      // live edges of the store during a contraction or compaction
  uint64_t store_list_cap = 0;

  // ---- profiling ----
  bool prof_on = false;
  bool capturing = false;                // launches are being recorded into a CUDA graph: no event timing
  std::vector<cudaEvent_t> prof_ev[3];   // [class] begin/end pairs: 0 ingest, 1 bucketing, 2 query
  size_t prof_used[3] = {0, 0, 0};
  uint64_t prof_launches[3] = {0, 0, 0};
  uint64_t launches_total = 0;
  uint64_t records_total = 0;
};

// Makes a device current for the duration of a call and restores the caller's.
struct GsDeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit GsDeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) { ok = false; return; }
    if (dev >= 0 && dev != prev) ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~GsDeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Frees every buffer a handle owns, then the handle.
void gs_free_graph(gs_graph* g);

enum GsProfClass { GS_PROF_INGEST = 0, GS_PROF_BUCKET = 1, GS_PROF_QUERY = 2 };

// Brackets a group of `launches` kernel launches of one class with CUDA events on stream s.
struct GsProfScope {
  gs_graph* g;
  int cls;
  long idx = -1;
  cudaStream_t s;
  GsProfScope(gs_graph* g_, int cls_, cudaStream_t s_, uint32_t launches);
  ~GsProfScope();
};

// Partial-support helpers implemented in the .cu files.
gs_status gs_ensure_ingest_scratch(gs_graph* g, uint64_t records);
// The page-locked staging ring (two slots) for host slices of up to `want` pairs, grown as needed up to
// min(max_batch_edges, 2^25); UINT64_MAX sizes it at that limit.
gs_status gs_ensure_pair_staging(gs_graph* g, uint64_t want = ~0ull);
// Sizes the single-level ingest scratch for batches of `edges` records, so that a later ingest of
// at most that many records allocates nothing (required while a stream is being captured).
gs_status gs_reserve_ingest(gs_graph* g, uint64_t edges);

// Ingest n edge records already on the device (interleaved pairs).  fixed_level < 0: every level
// the edge tags into (min-cut) or level 0 (connected components); >= 0: that level only.
gs_status gs_ingest_device_pairs(gs_graph* g, const uint32_t* d_pairs, uint64_t n, int fixed_level,
                                 cudaStream_t s);
// Directed per-vertex batches (already on the device).
gs_status gs_ingest_device_batches(gs_graph* g, uint32_t level, const uint32_t* d_srcs,
                                   const uint64_t* d_starts, const uint64_t* d_sizes,
                                   uint32_t nb, const uint32_t* d_dsts, cudaStream_t s,
                                   uint64_t max_records = 0);  // 0: read the record count back
// Device Boruvka on one level; forest edges stay in g->d_forest.
gs_status gs_boruvka(gs_graph* g, uint32_t level, uint32_t round0_col, cudaStream_t s);
// The same in two halves: the launch and the read-back of status words [0, 17) into pinned h_out
// (word 16: ingest error bits queued before the query), queued on s without waiting; then, once
// that work is done, the interpretation of those words.
gs_status gs_boruvka_enqueue(gs_graph* g, uint32_t level, uint32_t round0_col, cudaStream_t s, uint32_t* h_out);
gs_status gs_boruvka_finish(gs_graph* g, uint32_t level, const uint32_t* st);

// Eager DSU (gs_eager.cu).
gs_status gs_eager_enable(gs_graph* g, bool on, cudaStream_t s);
gs_status gs_eager_reset_empty(gs_graph* g, cudaStream_t s);           // the empty graph: valid, no forest
gs_status gs_eager_invalidate(gs_graph* g, cudaStream_t s);            // the next query runs Boruvka
gs_status gs_eager_ingest(gs_graph* g, const uint32_t* d_pairs, uint64_t n, cudaStream_t s);
gs_status gs_eager_state(gs_graph* g, cudaStream_t s, bool* valid);    // synchronizes
gs_status gs_eager_answer(gs_graph* g, cudaStream_t s);                // labels from the DSU
gs_status gs_eager_rebuild(gs_graph* g, cudaStream_t s);               // after a Boruvka query
gs_status gs_eager_forest(gs_graph* g, cudaStream_t s);                // the eager forest into d_forest

// Exact tier of the deep min-cut levels (gs_store.cu).
bool gs_store_active(const gs_graph* g);                               // tags can reach past the sketches
// After an ingest pass: when the store holds store_budget live edges or more and a sketch level is
// free, its lowest level becomes a sketch level (repeatedly); a store crowded by deleted edges is
// compacted.  Synchronizes.
gs_status gs_store_maintain(gs_graph* g, cudaStream_t s);
gs_status gs_store_ingest(gs_graph* g, const uint32_t* d_pairs, uint64_t n, cudaStream_t s);
gs_status gs_store_clear(gs_graph* g, cudaStream_t s);
gs_status gs_store_edges(gs_graph* g, uint32_t min_tag, std::vector<uint32_t>* out, cudaStream_t s);

// One independent graph of a Boruvka launch (gs_boruvka.cu).
struct GsBorTenant {
  uint64_t sk_off;      // bucket offset of the tenant's vertex-0 sketch from the launch's sketch base
  uint64_t csmix;       // checksum hash constant mix(B(seed))
  uint32_t vbase;       // first vertex of the tenant in the launch's vertex space
  uint32_t V, nb, bkt, ns;
  uint32_t round0_col;  // column sampled in round 0
};

struct GsBorLaunch {
  const GsBucket* sk = nullptr;
  const GsBorTenant* tenants = nullptr;  // device [T] when T > 1
  GsBorTenant t0{};                      // the tenant when T == 1
  const uint32_t* vtenant = nullptr;     // device [V] when T > 1
  uint32_t T = 1, V = 0, W = 0, max_rounds = 0;
  uint32_t vlo = 0;                      // vertices [vlo, V) take part
  uint32_t* parent = nullptr;
  uint32_t* size = nullptr;
  GsBucket* acc = nullptr;
  uint64_t* samp = nullptr;              // [V]
  uint32_t* roots = nullptr;             // [V]
  uint32_t* forest = nullptr;
  uint32_t forest_cap = 0;
  uint32_t* status = nullptr;            // 8 words: [0] errors [4] forest edges [5] running tenants [6,7] barrier
  uint32_t* tstate = nullptr;            // [T][4]: done, modified, rounds, out of samples
  uint64_t wait_ns = kGsDefaultWaitNs;   // grid-barrier wait limit
  // Only when every graph's vertex sketches XOR to zero (every update reached both endpoints): each
  // graph's largest component's merged column is taken as the XOR of the graph's vertices outside it,
  // so the accumulate phase never reads the largest components' own members.  `largest` is device
  // scratch of T 64-bit words.
  uint32_t complement = 0;
  unsigned long long* largest = nullptr;
};

// All Boruvka rounds of every tenant in one cooperative launch (queued on s, no host sync).
gs_status gs_boruvka_launch(const GsBorLaunch& L, cudaStream_t s);

// Exact global min cut (host), gs_mincut.cpp.
uint64_t gs_exact_min_cut_host(uint32_t V, const uint32_t* pairs, uint64_t m, uint8_t* side);

// R-MAT record generator shared by host and device (gs_gen.cu).
gs_status gs_gen_rmat_device(uint32_t log2_v, double a, double b, double c, double delete_frac,
                             uint64_t seed, uint64_t first, uint64_t n, uint32_t* d_pairs,
                             cudaStream_t s);
void gs_gen_rmat_host(uint32_t log2_v, double a, double b, double c, double delete_frac,
                      uint64_t seed, uint64_t first, uint64_t n, uint32_t* pairs);

GsTuning gs_tune_for(const GsGeom& geom, int num_sms);

// Everything one ingest pass over single-level sketches needs, with every scratch buffer supplied by
// the caller (the allocation-free entry point, gs_noalloc.cu).
struct GsScratchIngest {
  const uint32_t* pairs = nullptr;   // device, n interleaved pairs
  uint64_t n = 0;
  GsBucket* sketches = nullptr;      // device, [V][num_buckets]
  GsGeom geom{};
  const uint64_t* colmix = nullptr;  // device, num_columns + 1 constants
  uint32_t* status = nullptr;        // device, 16 words
  uint32_t* cnt = nullptr;           // device, V + 1
  uint32_t* off = nullptr;           // device, V + 1
  uint32_t* choff = nullptr;         // device, V + 1
  uint32_t* tile = nullptr;          // device, 2 * (ceil(V / 4096) + 1)
  uint32_t* bkt = nullptr;           // device, 4 * buckets + 2
  uint2* part = nullptr;             // device, records_cap
  uint32_t* nbr = nullptr;           // device, records_cap
  uint64_t records_cap = 0;
  uint32_t part_lb = 9;
  uint32_t part_buckets = 0;
  int num_sms = 148;
  uint32_t chunk = 1024;
  uint32_t warps = 4;
};

// Runs the bucketing passes and the sketch update on the buffers of `x` (no allocation).
gs_status gs_ingest_pairs_on_scratch(const GsScratchIngest& x, cudaStream_t s);
// Shared-memory bytes of one sketch-update block, for sizing checks by callers of the above.
size_t gs_scratch_ingest_smem_bytes(const GsGeom& geom, uint32_t warps);
