/*
 * gpusketch.h - C ABI of the B200 graph-stream sketching engine.
 *
 * Every entry point takes plain pointers and sizes, returns a gs_status and never
 * throws or exits.  The library owns all device memory; host pointers are borrowed
 * for the duration of a call.  A gs_graph handle is not thread-safe: use one thread
 * per handle or serialise calls.  Distinct handles may be used concurrently.
 *
 * Terms (the reference's domain vocabulary):
 *   vertex sketch   num_buckets Buckets {u64 alpha; u64 gamma} (16 B, packed) laid out as
 *                   num_columns columns of bkt_per_col buckets followed by one
 *                   deterministic bucket (reference include/bucket.h:7-12,
 *                   src/sketch.cpp:8-22,85-99).
 *   sketch set      [num_levels][num_vertices][num_buckets] Buckets in HBM.  A connected-
 *                   components graph has one level; a min-cut graph keeps one level per
 *                   sketched subgraph (reference src/mc_sketch_alg.cpp:93-122).
 *   edge record     one stream update (insert or delete) of the undirected edge {src,dst};
 *                   it XOR-toggles the edge id (min<<32)|max in both endpoint sketches
 *                   (reference src/cc_sketch_alg.cpp:154-160, src/util.cpp:45-51).
 *
 * Reference interfaces replaced (paths within the reference project):
 *   include/cuda_kernel.cuh:23-51     SketchParams, CudaKernel::sketchUpdate
 *   include/cuda_stream.h:146-276     CudaStream::process_batch / flush_buffers
 *   src/cc_gpu_sketch_alg.cpp:7-31    CCGPUSketchAlg::apply_update_batch / flush_buffers
 *   src/cc_sketch_alg.cpp:491-683     boruvka_emulation, connected_components, point_query,
 *                                     calc_spanning_forest, write_binary
 *   src/mc_sketch_alg.cpp:738-1002    k_boruvka_emulation, calc_disjoint_spanning_forests,
 *                                     calc_minimum_cut
 *   src/mc_gpu_sketch_alg.cpp:139-178 MCGPUSketchAlg::apply_update_batch (subgraph tagging)
 */
#ifndef GPUSKETCH_H_
#define GPUSKETCH_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_ABI_VERSION 1

typedef enum gs_status {
  GS_OK = 0,
  GS_ERR_BAD_ARG = 1,        /* invalid argument or out-of-range vertex id */
  GS_ERR_CUDA = 2,           /* CUDA runtime error (message in gs_last_error) */
  GS_ERR_OOM = 3,            /* device or pinned host allocation failed */
  GS_ERR_SKETCH_FAIL = 4,    /* Boruvka ran out of sketch columns (OutOfSamplesException) */
  GS_ERR_TIMEOUT = 5,        /* a bounded device-side wait gave up */
  GS_ERR_UPDATE_LOCKED = 6,  /* update while a query holds the sketches (UpdateLockedException) */
  GS_ERR_IO = 7,             /* file read/write failed */
  GS_ERR_INTERNAL = 8,       /* device-side consistency check failed */
  GS_ERR_NO_DEVICE = 9       /* no CUDA device or the kernels were not built for it */
} gs_status;

/* Bucket as stored in device memory and in the checkpoint file (include/bucket.h:7-12). */
typedef struct gs_bucket {
  uint64_t alpha; /* XOR of edge ids */
  uint64_t gamma; /* XOR of XXH3(edge id, seed) checksums */
} gs_bucket;

/* Sketch geometry derived exactly as the reference does (include/sketch.h:177-191,312-320,
 * src/sketch.cpp:24-30): num_samples = max(18, ceil(f*log2(V)/0.736965594)),
 * cols_per_sample = 1, bkt_per_col = ceil(log2(V(V-1)/2))+1 (bumped by one when a
 * multiple of 16), num_buckets = num_columns*bkt_per_col + 1. */
typedef struct gs_geometry {
  uint32_t num_vertices;
  uint32_t num_samples;
  uint32_t cols_per_sample;
  uint32_t num_columns;
  uint32_t bkt_per_col;
  uint32_t num_buckets;
  uint64_t bytes_per_vertex; /* num_buckets * 16 */
} gs_geometry;

/* Host-only sizing; replaces Sketch::calc_vector_length / calc_cc_samples /
 * calc_bkt_per_col (include/sketch.h:177-191,312-320). */
gs_status gs_geometry_for(uint32_t num_vertices, double sketches_factor, gs_geometry* out);

/* Host reference of the 8-byte XXH3_64bits_withSeed used for every column, checksum and
 * subgraph hash (include/types.h:8-9, include/bucket.h:54-63). */
uint64_t gs_hash64(uint64_t key, uint64_t seed);

typedef struct gs_graph_config {
  uint32_t num_vertices;   /* V; vertex ids are [0, V) */
  uint32_t num_levels;     /* 1 = connected-components graph; >1 = min-cut subgraph levels */
  uint64_t seed;           /* sketch seed; column c hashes with seed+5c, checksum with seed */
  double sketches_factor;  /* CCAlgConfiguration::sketches_factor (<=0 means 1) */
  double batch_factor;     /* CCAlgConfiguration::batch_factor (<=0 means 1) */
  uint32_t num_subgraphs;  /* min-cut tag bound L: level = ctz(XXH3(e,seed) | 1<<(L-1)); 0 = num_levels */
  int32_t device;          /* CUDA device ordinal; -1 = current device */
  uint64_t max_batch_edges;/* edges per internal ingest pass; 0 = library default (2^27) */
} gs_graph_config;

typedef struct gs_graph gs_graph;

/* Allocates zeroed sketches for every level (CCSketchAlg / MCSketchAlg constructors,
 * src/cc_sketch_alg.cpp:11-55, src/mc_sketch_alg.cpp:16-40,93-122). */
gs_status gs_graph_create(const gs_graph_config* cfg, gs_graph** out);
gs_status gs_graph_destroy(gs_graph* g);
gs_status gs_graph_geometry(const gs_graph* g, gs_geometry* out);
/* Zeroes every sketch of the set (Sketch::zero_contents over all vertices, src/sketch.cpp:102-108). */
gs_status gs_clear(gs_graph* g);
/* Makes the handle launch on `cuda_stream` (cudaStream_t; NULL restores its own stream), so the
 * caller's CUDA events on that stream bracket the handle's kernels. */
gs_status gs_graph_set_stream(gs_graph* g, void* cuda_stream);
/* Updates per worker batch the reference would buffer: bucket_array_bytes/4*batch_factor
 * (include/cc_sketch_alg.h:147-151). */
uint64_t gs_desired_updates_per_batch(const gs_graph* g);

/* Ingest n edge records given as interleaved uint32 pairs [src0,dst0,src1,dst1,...].
 * Each record toggles edge {src,dst} in both endpoint sketches of every level the edge
 * tags into (one level for connected-components graphs).  Self-loops are no-ops, as in
 * the reference where the two updates of sketch src cancel.  pairs_on_device != 0 means
 * `pairs` is a device pointer; otherwise it is host memory (pinned or pageable) staged
 * through the library's pinned ring.  `cuda_stream` (cudaStream_t, may be NULL) orders the
 * work after the caller's stream.  Replaces the GPU worker path
 * GraphSketchDriver::batch_callback -> CCGPUSketchAlg::apply_update_batch ->
 * CudaStream::process_batch -> CudaKernel::sketchUpdate (include/graph_sketch_driver.h:204-208,
 * src/cc_gpu_sketch_alg.cpp:7-19, include/cuda_stream.h:146-202, src/cuda_kernel.cu:242-257). */
gs_status gs_ingest_pairs(gs_graph* g, const uint32_t* pairs, uint64_t n, int pairs_on_device,
                          void* cuda_stream);

/* Allocates now what host input needs - the page-locked staging ring for slices of up to `records`
 * records (at most min(max_batch_edges, 2^25)) and the stream-file decode buffer - instead of at the
 * first host ingest; page-locking hundreds of megabytes takes tens of milliseconds.  Library extension
 * (the reference's CCGPUSketchAlg constructor sets up its CudaStream buffers the same way,
 * include/cc_gpu_sketch_alg.h:36-95). */
gs_status gs_prepare_host_input(gs_graph* g, uint64_t records);

/* gs_ingest_pairs without waiting for host input to be copied: the call queues the copies and the
 * ingest and returns.  For page-locked host memory it returns at once and the buffer stays in use until
 * the handle's queued work is done (gs_synchronize, gs_query_wait, or any synchronous query): the caller
 * must neither free nor change it before then.  Pageable memory is still staged through the pinned
 * ring and may be reused when the call returns.  The copies wait for their staging slots on the
 * device, so copies of the next phase's records proceed while a query queued with
 * gs_connected_components_async runs.  Device input behaves as in gs_ingest_pairs.  Library extension
 * (the reference's CudaStream waits for each buffer, include/cuda_stream.h:146-202). */
gs_status gs_ingest_pairs_async(gs_graph* g, const uint32_t* pairs, uint64_t n, int pairs_on_device,
                                void* cuda_stream);

/* Edge records [first, first+count) of a binary stream file in the reference's format (a header
 * {u32 num_vertices, u64 num_updates}, then packed 9-byte records {u8 type, u32 src, u32 dst}; the
 * StreamingUtilities BinaryFileStream read by the reference's tools and tests).  count may exceed the
 * records left (UINT64_MAX: to the end).  The file is read in slices by several threads straight into
 * the library's page-locked ring, copied to the device as raw records and decoded there; the read and
 * copy of slice k+1 overlap the ingest of slice k.  Every record toggles its edge whatever its type
 * byte, as in the reference's sketch update.  *ingested (may be NULL) receives the record count.
 * GS_ERR_IO on an unreadable or truncated file, GS_ERR_BAD_ARG when the file's vertex count exceeds
 * the graph's.  Replaces the reader threads of GraphSketchDriver::process_stream_until
 * (include/graph_sketch_driver.h:141-191) for file streams. */
gs_status gs_ingest_stream_file(gs_graph* g, const char* path, uint64_t first, uint64_t count,
                                uint64_t* ingested);

/* Same as gs_ingest_pairs with separate src / dst arrays (device arrays are interleaved on the device). */
gs_status gs_ingest_edges(gs_graph* g, const uint32_t* src, const uint32_t* dst, uint64_t n,
                          int on_device, void* cuda_stream);

/* The reference's per-vertex batch form: batch b XORs edges (srcs[b], dsts[starts[b] + i]),
 * i < sizes[b], into the sketch of srcs[b] ONLY, at sketch level `level`
 * (CCSketchAlg::apply_update_batch, src/cc_sketch_alg.cpp:133-145;
 * CudaKernel::sketchUpdate inputs, include/cuda_kernel.cuh:46). */
gs_status gs_ingest_vertex_batches(gs_graph* g, uint32_t level, const uint32_t* srcs,
                                   const uint64_t* starts, const uint64_t* sizes,
                                   uint32_t num_batches, const uint32_t* dsts,
                                   uint64_t num_dsts, int on_device, void* cuda_stream);

/* Waits until every queued update is applied (CCGPUSketchAlg::flush_buffers,
 * src/cc_gpu_sketch_alg.cpp:21-31; MCGPUSketchAlg::apply_flush_updates). */
gs_status gs_synchronize(gs_graph* g);

/* Device Boruvka emulation on sketch level `level` (CCSketchAlg::connected_components,
 * src/cc_sketch_alg.cpp:491-584).  labels (host, length V, may be NULL) receives the minimum
 * vertex id of each vertex's component; num_cc and rounds may be NULL.  Returns
 * GS_ERR_SKETCH_FAIL when the sketch runs out of columns. */
gs_status gs_connected_components(gs_graph* g, uint32_t level, uint32_t* labels, uint32_t* num_cc,
                                  uint32_t* rounds);

/* connected_components() queued without waiting for it (library extension): the query sees every
 * update queued before it and none queued after it, so the caller can queue the next phase's ingest
 * (gs_ingest_pairs_async) while it runs.  gs_query_wait collects the answer; until then no other query
 * may be made on the handle (GS_ERR_BAD_ARG).  The first call allocates page-locked space for the
 * answer (V labels).  With the eager DSU on, the answer is computed at once. */
gs_status gs_connected_components_async(gs_graph* g, uint32_t level);
/* Waits for the query queued by gs_connected_components_async and returns what gs_connected_components
 * would have returned for it: labels (host, length V, may be NULL), num_cc and rounds (may be NULL),
 * GS_ERR_SKETCH_FAIL when the sketches ran out of columns, GS_ERR_BAD_ARG when an ingest queued before
 * the query had skipped out-of-range records. */
gs_status gs_query_wait(gs_graph* g, uint32_t* labels, uint32_t* num_cc, uint32_t* rounds);

/* CCSketchAlg::point_query (src/cc_sketch_alg.cpp:630-672). */
gs_status gs_point_query(gs_graph* g, uint32_t a, uint32_t b, int* connected);

/* Spanning forest found by the last Boruvka run on `level` (calc_spanning_forest,
 * src/cc_sketch_alg.cpp:586-595).  edges (host) holds 2*(V-1) uint32 as (src<dst) pairs. */
gs_status gs_spanning_forest(gs_graph* g, uint32_t level, uint32_t* edges, uint64_t* num_edges);

/* k edge-disjoint spanning forests of sketch level `level`: after each forest its edges are
 * XOR-deleted from the level's sketches, and all are re-inserted at the end
 * (MCSketchAlg::calc_disjoint_spanning_forests / filter_sf_edges,
 * src/mc_sketch_alg.cpp:837-919).  edges (host) holds k*2*(V-1) uint32, forest f starting at
 * offset f*2*(V-1); forest_sizes[f] receives its edge count. */
gs_status gs_disjoint_spanning_forests(gs_graph* g, uint32_t level, uint32_t k, uint32_t* edges,
                                       uint64_t* forest_sizes);

/* Min-cut driver of the reference's tools/min_cut.cu:208-252: for level g = 0,1,... take k
 * disjoint spanning forests, compute the exact minimum cut of their union, and stop at the
 * first level whose cut is < k.  When no sketched level does and tags can pass the sketches
 * (num_subgraphs > the sketched levels), the first unsketched level answers from the exact tier (see
 * gs_edge_store_edges) with the exact min cut of all its edges, whatever its value; otherwise
 * the last sketched level answers.
 * value = cut * 2^g.  side (host, length V, may be NULL) receives 1 for vertices on one side. */
gs_status gs_min_cut(gs_graph* g, uint32_t k, uint64_t* value, uint32_t* level_found,
                     uint64_t* cut_at_level, uint8_t* side);

/* Exact global minimum cut of an undirected multigraph given as uint32 pairs (host).
 * Replaces the VieCut call of MCSketchAlg::calc_minimum_cut (src/mc_sketch_alg.cpp:966-1002). */
gs_status gs_exact_min_cut(uint32_t num_vertices, const uint32_t* pairs, uint64_t num_edges,
                           uint64_t* value, uint8_t* side);

/* The exact tier of a min-cut graph (EdgeStore, src/edge_store.cpp:60-300; get_edges): edges whose
 * subgraph tag reaches the sketched levels are also kept exactly on the device, with each toggle
 * flipping their presence; gs_min_cut answers from them when no sketched level certifies a cut below
 * k.  Writes the present edges with tag >= min_tag (sorted by edge id, at most `capacity`) and their
 * count to *num_edges.  Empty when num_subgraphs <= the sketched levels (no tag passes the sketches). */
gs_status gs_edge_store_edges(gs_graph* g, uint32_t min_tag, uint32_t* edges, uint64_t capacity,
                              uint64_t* num_edges);

/* Makes the exact tier adaptive, as the reference's EdgeStore (src/edge_store.cpp:60-300,
 * include/mc_gpu_sketch_alg.h:168-230): the graph starts with `initial_sketch_levels` sketched levels
 * (0 = every edge kept exactly) of its num_levels, and edges whose tag reaches the sketched levels are
 * kept exactly.  After each ingest pass, when the tier holds at least store_bytes / 16 present edges
 * (the reference's bound: sketch_bytes / 8 per directed adjacency entry, two per edge; 0 = one sketch
 * level's bytes) and a level is free, its lowest level becomes a sketch level: the stored edges of
 * that level and above are XORed into it and only deeper ones stay exact.  gs_min_cut then walks the
 * levels sketched at query time and answers the next one from the exact tier.  Only on a min-cut graph
 * (num_subgraphs > 1) with no ingest since creation or gs_clear; gs_clear returns to the initial
 * levels.  Edges whose tag would be num_subgraphs - 1 or more are tagged num_subgraphs - 1, where the
 * reference's all-exact start tags them num_subgraphs (src/edge_store.cpp:51): both exceed every level
 * a graph can sketch. */
gs_status gs_graph_set_edge_store(gs_graph* g, uint32_t initial_sketch_levels, uint64_t store_bytes);
/* Levels sketched now (MCGPUSketchAlg::get_num_sketch_graphs) and contractions so far. */
gs_status gs_graph_sketched_levels(const gs_graph* g, uint32_t* levels, uint64_t* contractions);

/* Copy vertex sketches [first, first+count) of `level` to / from host memory in the
 * contiguous [vertex][num_buckets] Bucket layout of Sketch::serialize
 * (src/sketch.cpp:204-206). */
gs_status gs_download_sketches(gs_graph* g, uint32_t level, uint32_t first_vertex, uint32_t count,
                               void* host_out);
gs_status gs_upload_sketches(gs_graph* g, uint32_t level, uint32_t first_vertex, uint32_t count,
                             const void* host_in);

/* Checkpoint in the reference's format: [u64 seed][u32 V][f64 sketches_factor] then
 * V*num_buckets Buckets of level 0 (CCSketchAlg::write_binary, src/cc_sketch_alg.cpp:674-683;
 * construct_from_serialized_data, :57-91). */
gs_status gs_write_binary(gs_graph* g, const char* path);
gs_status gs_read_binary(const char* path, int32_t device, gs_graph** out);

/* ---- eager DSU / cached connectivity ----
 * With the eager DSU on, every ingest keeps a device DSU and spanning forest of the stream next to
 * the sketches, and gs_connected_components answers from them - without Boruvka - until a record may
 * have deleted a forest edge; the next query then runs Boruvka and rebuilds them from its forest
 * (CCSketchAlg::pre_insert, src/cc_sketch_alg.cpp:106-131; connected_components :542-549).  Records
 * of a batch are applied concurrently, so a batch that toggles an edge it has just made a forest
 * edge also invalidates.  Connected-components graphs only; off by default (the reference's
 * NO_EAGER_DSU build), because streams with frequent deletions pay the passes and rarely profit.
 * gs_ingest_vertex_batches and gs_upload_sketches invalidate; gs_clear resets to the empty graph. */
gs_status gs_set_eager_dsu(gs_graph* g, int enable);
/* has_cached_query(CONNECTIVITY) (include/cc_sketch_alg.h:185-191): 1 when the next
 * gs_connected_components will be answered from the eager DSU.  Synchronizes the handle. */
gs_status gs_has_cached_query(gs_graph* g, int* cached);

/* ---- bounded device-side waits ----
 * Every wait of a device kernel on other blocks (the grid barriers of the persistent Boruvka kernel)
 * gives up after a limit, sets a device error bit and lets the kernel return, so a wait that cannot
 * end leaves the context usable: the query then fails with GS_ERR_TIMEOUT and the next query starts
 * from scratch.  Sets that limit for this handle's queries (summed sleep time of one wait; default
 * about one second; 0 restores the default).  Library extension without a reference counterpart;
 * the tests set a limit far below one barrier's normal wait to make a wait run out. */
gs_status gs_set_device_wait_limit(gs_graph* g, uint64_t nanoseconds);

/* ---- tuning (set by the autotuner, gpusketch_b200/autotune.py) ---- */
typedef struct gs_tuning {
  uint32_t chunk;            /* records per sketch-update work item (>= 32) */
  uint32_t warps_per_block;  /* warps per sketch-update block (1..16; the packed layout runs at most 12) */
  uint32_t reg_depth;        /* bucket depths each lane keeps in registers (0..3); 0 on a sketch of at
                                most 32 columns selects the packed layout, in which lanes left over by
                                the columns take columns of further records */
  uint32_t reserved;
} gs_tuning;
/* Reads / replaces the launch parameters of the sketch-update kernel.  Results never depend on them.
 * Library extension without a reference counterpart (the reference hard-codes 1024 threads and
 * 540 batches per launch, include/cc_gpu_sketch_alg.h:14-33). */
gs_status gs_get_tuning(const gs_graph* g, gs_tuning* out);
gs_status gs_set_tuning(gs_graph* g, const gs_tuning* t);

/* ---- profiling (per-handle CUDA-event timing on the stream each kernel is launched on) ---- */
typedef struct gs_profile {
  uint64_t ingest_launches;  /* sketch-update kernel launches */
  double ingest_ms;          /* their summed event-timed duration */
  uint64_t bucket_launches;  /* endpoint-bucketing kernel launches (count, scan, scatter) */
  double bucket_ms;
  uint64_t query_launches;   /* Boruvka kernel launches */
  double query_ms;
  uint64_t kernel_launches;  /* every kernel this handle launched */
  uint64_t records_ingested; /* edge records consumed by the ingest path */
} gs_profile;

/* Resets the counters; when `enable` is non-zero, brackets each kernel group with CUDA events.
 * Library extension without a reference counterpart (the reference times with std::chrono,
 * include/cuda_stream.h:286-291). */
gs_status gs_profile_enable(gs_graph* g, int enable);
/* Waits for queued work and returns the counters accumulated since gs_profile_enable. */
gs_status gs_profile_read(gs_graph* g, gs_profile* out);

/* ---- allocation-free ingest ----
 * No counterpart in the reference.  For callers that cannot allocate device memory because another
 * allocator owns it (a framework's caching allocator, an embedded runtime that forbids allocation
 * after start-up).  XORs n edge records (device pointer, interleaved uint32 pairs) into the caller's
 * device sketches of a connected-components graph, laid out [V][num_buckets] gs_bucket as
 * gs_geometry_for(num_vertices, sketches_factor) sizes them; the result equals gs_ingest_pairs on a
 * gs_graph with the same seed and factor.  Calls no allocator: all scratch is one static device array
 * of about 2.3 MB that every GPU loading the library holds until exit; each call looks up the array's
 * device address on the current device.  The array is shared by all calls and keeps the last call's
 * contents, so calls that overlap on the GPU race.  Rejects num_vertices outside
 * [2, GS_NOALLOC_MAX_VERTICES] and n > GS_NOALLOC_MAX_EDGES with GS_ERR_BAD_ARG before touching the
 * sketches.  Runs on `cuda_stream` (may be NULL) on the current device and is synchronous: it waits
 * for that stream to apply the update and check the device error word, so it must not be called while
 * the stream is being captured into a CUDA graph.  When a record names a vertex >= num_vertices the
 * call returns GS_ERR_BAD_ARG after applying every other record of the call (only the out-of-range
 * records are skipped), so a caller that retries must not resend the records that were applied. */
#define GS_NOALLOC_MAX_VERTICES 65536u
#define GS_NOALLOC_MAX_EDGES 65536u
gs_status gs_ingest_pairs_noalloc(uint32_t num_vertices, uint64_t seed, double sketches_factor,
                                  const uint32_t* pairs, uint64_t n, gs_bucket* sketches,
                                  void* cuda_stream);

/* ---- multi-tenant engine: many independent connected-components graphs on one GPU ----
 *
 * No single reference counterpart: the reference runs one CCSketchAlg per process.  Each tenant is
 * a graph with its own vertex count, seed and sketches_factor whose sketches are bit-identical to
 * a gs_graph (equivalently a reference CCSketchAlg) with the same parameters fed the same records;
 * tenants never share a bucket, so a tenant's sketches and answers do not depend on the others.
 *
 *   tenant sketches  [V][num_buckets] gs_bucket inside the engine's device arena (first fit).
 *   vertex space     each tenant owns V consecutive ids of the engine's vertex space.
 *   slice            a run of records of one tenant inside one ingest call.
 *
 * Admission: gs_engine_add_tenant fails with GS_ERR_OOM when the arena, the vertex space or the
 * tenant slots cannot hold the tenant; removing tenants frees their space.  An engine handle is
 * not thread-safe. */
typedef struct gs_engine gs_engine;

typedef struct gs_engine_config {
  uint64_t sketch_budget_bytes;  /* device arena for tenant sketches (the admission limit) */
  uint32_t max_tenants;          /* tenant slots (1..4096) */
  uint32_t max_vertices;         /* engine vertex space: total V over live tenants */
  uint32_t max_tenant_vertices;  /* largest V of one tenant (sizes the Boruvka scratch) */
  int32_t device;                /* CUDA device ordinal; < 0 = current device */
  uint64_t max_batch_edges;      /* records per internal ingest pass (0 = 2^25) */
} gs_engine_config;

gs_status gs_engine_create(const gs_engine_config* cfg, gs_engine** out);
gs_status gs_engine_destroy(gs_engine* e);
/* Device bytes the sketches of one tenant take (what admission charges). */
gs_status gs_engine_tenant_bytes(uint32_t num_vertices, double sketches_factor, uint64_t* bytes);
/* Admits a tenant with zeroed sketches (CCSketchAlg(num_vertices, seed, config) with
 * config.sketches_factor; src/cc_sketch_alg.cpp:11-55).  GS_ERR_OOM: not admitted now. */
gs_status gs_engine_add_tenant(gs_engine* e, uint32_t num_vertices, uint64_t seed, double sketches_factor,
                               uint32_t* tenant);
gs_status gs_engine_remove_tenant(gs_engine* e, uint32_t tenant);
/* Zeroes one tenant's sketches (Sketch::zero_contents over its vertices, src/sketch.cpp:102-108). */
gs_status gs_engine_clear_tenant(gs_engine* e, uint32_t tenant);
/* Sketch bytes in use by live tenants, the arena size, and the live tenant count. */
gs_status gs_engine_memory(const gs_engine* e, uint64_t* used, uint64_t* capacity, uint32_t* live_tenants);
gs_status gs_engine_set_stream(gs_engine* e, void* cuda_stream);
/* Ingests num_slices slices in one pass: slice i is records [slice_offsets[i], slice_offsets[i+1])
 * of `pairs` (interleaved tenant-local uint32 vertex ids) for tenant slice_tenants[i].  Per tenant
 * this is gs_ingest_pairs; the bucketing and the sketch update of all slices run as one launch
 * each.  pairs is a device pointer when pairs_on_device != 0; the slice tables are host arrays.  A
 * record naming a vertex >= its tenant's V is skipped and reported as GS_ERR_BAD_ARG by the next
 * gs_engine_synchronize or query. */
gs_status gs_engine_ingest(gs_engine* e, const uint32_t* slice_tenants, const uint64_t* slice_offsets,
                           uint32_t num_slices, const uint32_t* pairs, int pairs_on_device, void* cuda_stream);
/* Gather form for serving: slice i is slice_counts[i] records at HOST address slice_pairs[i] for
 * tenant slice_tenants[i]; the slices are coalesced into one bucketing pass and one sketch update.
 * Page-locked slices are copied to the device directly, others through the pinned staging ring.
 * Returns once the caller's buffers may be reused; the device work may still be running (the copy
 * of the next call overlaps it). */
gs_status gs_engine_ingest_slices(gs_engine* e, uint32_t num_slices, const uint32_t* slice_tenants,
                                  const uint64_t* slice_counts, const uint32_t* const* slice_pairs,
                                  void* cuda_stream);
gs_status gs_engine_synchronize(gs_engine* e);
/* connected_components() of `count` distinct tenants in one device Boruvka launch.  labels
 * (host, may be NULL) receives each listed tenant's V labels back to back in list order, each the
 * smallest tenant-local vertex id of its component; num_cc[i] and rounds[i] (may be NULL) are the
 * component count and Boruvka rounds of tenants[i].  GS_ERR_SKETCH_FAIL when a listed tenant ran
 * out of samples (OutOfSamplesException); the others' results are still written. */
gs_status gs_engine_connected_components(gs_engine* e, const uint32_t* tenants, uint32_t count, uint32_t* labels,
                                         uint32_t* num_cc, uint32_t* rounds);
/* One phase of a batched workload: ingest slices of DEVICE-resident records (as gs_engine_ingest,
 * at most 2^25 records) and then answer connected_components() for `query_count` tenants (as
 * gs_engine_connected_components without labels; query_count may be 0).  With
 * GS_PHASE_CUDA_GRAPH in `flags` the phase's device work - slice-table upload, endpoint bucketing,
 * sketch update, the persistent Boruvka kernel and the result read-back - is recorded into one CUDA
 * graph and launched as a whole; a phase with the same sequence of steps as the previous one
 * updates that graph's parameters in place instead of instantiating a new one.  Returns after
 * the phase finished. */
#define GS_PHASE_CUDA_GRAPH 1
gs_status gs_engine_phase(gs_engine* e, const uint32_t* slice_tenants, const uint64_t* slice_offsets,
                          uint32_t num_slices, const uint32_t* pairs, const uint32_t* query_tenants,
                          uint32_t query_count, uint32_t* num_cc, uint32_t* rounds, int flags);
/* CUDA graphs instantiated and launched by gs_engine_phase so far. */
gs_status gs_engine_graph_stats(const gs_engine* e, uint64_t* graphs_built, uint64_t* graph_launches);
gs_status gs_engine_tenant_geometry(const gs_engine* e, uint32_t tenant, gs_geometry* out);
/* Tenant sketches of vertices [first, first+count) to host memory, in the write_binary layout. */
gs_status gs_engine_download_sketches(gs_engine* e, uint32_t tenant, uint32_t first, uint32_t count,
                                      gs_bucket* out);
/* Per-tenant checkpoint in the reference's write_binary format (src/cc_sketch_alg.cpp:57-91);
 * gs_read_binary reloads it as a gs_graph. */
gs_status gs_engine_write_binary(gs_engine* e, uint32_t tenant, const char* path);
gs_status gs_engine_get_tuning(const gs_engine* e, gs_tuning* out);
gs_status gs_engine_set_tuning(gs_engine* e, const gs_tuning* t);
gs_status gs_engine_profile_enable(gs_engine* e, int enable);
gs_status gs_engine_profile_read(gs_engine* e, gs_profile* out);

/* Last error message of the calling thread ("" when none). */
const char* gs_last_error(void);

/* ---- seeded synthetic streams (test and benchmark inputs; not reference code) ---- */

/* Erdos-Renyi G(V, p) edges in shuffled order, then a `delete_frac` share deleted and a
 * `reinsert_frac` share of those re-inserted.  Host-side; writes at most `capacity` pairs
 * and returns the record count in *n. */
gs_status gs_gen_er_stream(uint32_t num_vertices, double p, uint64_t seed, double delete_frac,
                           double reinsert_frac, uint32_t* pairs, uint64_t capacity, uint64_t* n);

/* R-MAT(a,b,c) stream over 2^log2_v vertices, records [first, first+n) of the counter-based
 * stream with a `delete_frac` share of records deleting an earlier inserted edge.  Runs on
 * the device when pairs_on_device != 0 (pairs is a device pointer), else on the host. */
gs_status gs_gen_rmat_stream(uint32_t log2_v, double a, double b, double c, double delete_frac,
                             uint64_t seed, uint64_t first, uint64_t n, uint32_t* pairs,
                             int pairs_on_device, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* GPUSKETCH_H_ */
