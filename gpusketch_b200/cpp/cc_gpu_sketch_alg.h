// cc_gpu_sketch_alg.h - CCGPUSketchAlg drop-in: the reference's connected-components algorithm
// interface (include/cc_sketch_alg.h:65-261, include/cc_gpu_sketch_alg.h:8-110) over the C ABI.
//
// The sketches live on the GPU for the lifetime of the object.  Worker-thread batches handed to
// apply_update_batch (thread-safe, as the driver contract requires, include/graph_sketch_driver.h:49-52)
// are buffered per call site and shipped in bulk through gs_ingest_vertex_batches, the way the
// reference's CudaStream gathers ~540 batches per kernel launch (include/cc_gpu_sketch_alg.h:20).
// Bulk edge records (the device-bucketed path) go through ingest_records.
#pragma once

#include <chrono>
#include <iostream>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpusketch_types.h"

class CCGPUSketchAlg {
 public:
  CCGPUSketchAlg(node_id_t num_vertices, size_t seed, CCAlgConfiguration config = CCAlgConfiguration(),
                 int device = -1)
      : num_vertices(num_vertices), seed(seed), config(config) {
    gs_graph_config cfg{};
    cfg.num_vertices = num_vertices;
    cfg.num_levels = 1;
    cfg.seed = seed;
    cfg.sketches_factor = config.get_sketches_factor();
    cfg.batch_factor = config.get_batch_factor();
    cfg.device = device;
    gs_throw_if(gs_graph_create(&cfg, &g), "gs_graph_create");
    flush_at = 540 * get_desired_updates_per_batch();
  }

  // The reference's constructor (include/cc_gpu_sketch_alg.h:36, called by tools/cuda_process_stream.cu:126):
  // the sketch seed comes from the SketchParams; the geometry is derived from num_nodes and
  // config.sketches_factor, which gives the sizes the tools compute into the SketchParams.  num_updates
  // sizes the host staging; num_threads worker threads may call apply_update_batch.
  CCGPUSketchAlg(node_id_t num_nodes, size_t num_updates, int num_threads, SketchParams sketch_params,
                 CCAlgConfiguration config = CCAlgConfiguration())
      : CCGPUSketchAlg(num_nodes, sketch_params.seed, config) {
    num_host_threads = num_threads > 0 ? num_threads : 1;
    // the stream's records arrive from the host: set up the page-locked staging now, as the
    // reference sets up its CudaStream buffers here
    gs_throw_if(gs_prepare_host_input(g, num_updates), "gs_prepare_host_input");
    gs_geometry geo{};
    gs_graph_geometry(g, &geo);
    if ((sketch_params.num_buckets && sketch_params.num_buckets != geo.num_buckets) ||
        (sketch_params.num_columns && sketch_params.num_columns != geo.num_columns))
      throw std::invalid_argument("SketchParams geometry differs from the one num_nodes and sketches_factor give");
  }

  ~CCGPUSketchAlg() { gs_graph_destroy(g); }
  CCGPUSketchAlg(const CCGPUSketchAlg&) = delete;
  CCGPUSketchAlg& operator=(const CCGPUSketchAlg&) = delete;

  // construct_from_serialized_data (src/cc_sketch_alg.cpp:57-70)
  static CCGPUSketchAlg* construct_from_serialized_data(const std::string& input_file,
                                                        CCAlgConfiguration config = CCAlgConfiguration()) {
    gs_graph* h = nullptr;
    gs_throw_if(gs_read_binary(input_file.c_str(), -1, &h), "gs_read_binary");
    gs_geometry geo{};
    gs_graph_geometry(h, &geo);
    return new CCGPUSketchAlg(h, geo.num_vertices, config);
  }

  // ---- driver contract (include/graph_sketch_driver.h:28-69) ----
  void allocate_worker_memory(size_t num_workers) { (void)num_workers; }
  size_t get_desired_updates_per_batch() { return gs_desired_updates_per_batch(g); }
  node_id_t get_num_vertices() { return num_vertices; }
  // With set_eager_dsu(true) the library keeps the DSU current on every ingested edge record, so
  // pre_insert has nothing left to do; has_cached_query reports whether connected_components() will
  // be answered without Boruvka (include/cc_sketch_alg.h:185-191).
  void pre_insert(GraphUpdate, int = 0) {}
  bool has_cached_query(int query_code) {
    if (query_code != CONNECTIVITY) return false;
    int cached = 0;
    gs_throw_if(gs_has_cached_query(g, &cached), "gs_has_cached_query");
    return cached != 0;
  }
  void set_eager_dsu(bool on) { gs_throw_if(gs_set_eager_dsu(g, on ? 1 : 0), "gs_set_eager_dsu"); }
  void print_configuration() { std::cout << config << std::endl; }

  // Each worker (thr_id, one thread each as the driver contract has it) fills a buffer of its own, as
  // the reference gives every worker its own CudaStream (include/cc_gpu_sketch_alg.h:63-67); a full
  // buffer is shipped under the handle's lock while the other workers keep filling theirs.
  void apply_update_batch(int thr_id, node_id_t src_vertex, const std::vector<node_id_t>& dst_vertices) {
    if (update_locked) throw UpdateLockedException();
    WorkerBuffer& b = worker(thr_id);
    Batches full;
    {
      std::lock_guard<std::mutex> wl(b.mtx);
      b.q.srcs.push_back(src_vertex);
      b.q.starts.push_back(b.q.dsts.size());
      b.q.sizes.push_back(dst_vertices.size());
      b.q.dsts.insert(b.q.dsts.end(), dst_vertices.begin(), dst_vertices.end());
      if (b.q.dsts.size() < flush_at) return;
      std::swap(full, b.q);
    }
    // the worker's lock is released before the handle's: flush_buffers takes them in the other order
    std::lock_guard<std::mutex> lk(mtx);
    ship(full);
  }

  // CCGPUSketchAlg::flush_buffers (src/cc_gpu_sketch_alg.cpp:21-31)
  void flush_buffers() {
    std::lock_guard<std::mutex> lk(mtx);
    for (auto& b : workers) {
      Batches q;
      {
        std::lock_guard<std::mutex> wl(b.mtx);
        std::swap(q, b.q);
      }
      ship(q);
    }
    gs_throw_if(gs_synchronize(g), "gs_synchronize");
  }

  // CCSketchAlg::update (src/cc_sketch_alg.cpp:154-160): both endpoint sketches
  void update(GraphUpdate upd) {
    uint32_t p[2] = {upd.edge.src, upd.edge.dst};
    ingest_records(p, 1);
  }

  // n edge records as interleaved (src, dst) pairs in host memory
  void ingest_records(const uint32_t* pairs, size_t n) {
    std::lock_guard<std::mutex> lk(mtx);
    gs_throw_if(gs_ingest_pairs(g, pairs, n, 0, nullptr), "gs_ingest_pairs");
  }

  // records [first, first+count) of a binary stream file, read by the library (gs_ingest_stream_file)
  void ingest_stream_file(const std::string& path, edge_id_t first, edge_id_t count) {
    std::lock_guard<std::mutex> lk(mtx);
    gs_throw_if(gs_ingest_stream_file(g, path.c_str(), first, count, nullptr), "gs_ingest_stream_file");
  }

  // CCGPUSketchAlg::display_time (src/cc_gpu_sketch_alg.cpp:34-75): what the device path did so far
  void display_time() {
    gs_profile p{};
    gs_throw_if(gs_profile_read(g, &p), "gs_profile_read");
    std::cout << "Device ingest: " << p.records_ingested << " edge records, " << p.ingest_launches
              << " sketch-update launches, " << p.kernel_launches << " kernel launches\n";
  }

  // ---- queries (src/cc_sketch_alg.cpp:542-683) ----
  ConnectedComponents connected_components() {
    flush_buffers();
    std::vector<node_id_t> labels(num_vertices);
    uint32_t ncc = 0, rounds = 0;
    cc_alg_start = std::chrono::steady_clock::now();
    gs_throw_if(gs_connected_components(g, 0, labels.data(), &ncc, &rounds), "gs_connected_components");
    cc_alg_end = std::chrono::steady_clock::now();
    last_query_rounds = rounds;
    return ConnectedComponents(std::move(labels));
  }

  bool point_query(node_id_t a, node_id_t b) {
    flush_buffers();
    int c = 0;
    gs_throw_if(gs_point_query(g, a, b, &c), "gs_point_query");
    return c != 0;
  }

  SpanningForest calc_spanning_forest() {
    flush_buffers();
    std::vector<uint32_t> e(2 * (size_t)num_vertices);
    uint64_t n = 0;
    gs_throw_if(gs_spanning_forest(g, 0, e.data(), &n), "gs_spanning_forest");
    return SpanningForest(to_edges(e.data(), n));
  }

  std::vector<SpanningForest> calc_disjoint_spanning_forests(size_t k) {
    flush_buffers();
    const size_t stride = 2 * (size_t)(num_vertices - 1);
    std::vector<uint32_t> e(k * stride);
    std::vector<uint64_t> sizes(k);
    gs_throw_if(gs_disjoint_spanning_forests(g, 0, (uint32_t)k, e.data(), sizes.data()),
                "gs_disjoint_spanning_forests");
    std::vector<SpanningForest> out;
    for (size_t f = 0; f < k; f++) out.emplace_back(to_edges(e.data() + f * stride, sizes[f]));
    return out;
  }

  void write_binary(const std::string& filename) {
    flush_buffers();
    gs_throw_if(gs_write_binary(g, filename.c_str()), "gs_write_binary");
  }

  // getters (include/cc_sketch_alg.h:256-260)
  size_t get_seed() { return seed; }
  size_t max_rounds() {
    gs_geometry geo{};
    gs_graph_geometry(g, &geo);
    return geo.num_samples;
  }
  bool get_update_locked() { return update_locked; }
  gs_graph* handle() { return g; }

  size_t last_query_rounds = 0;
  // time hooks of the last connected_components() (include/cc_sketch_alg.h:252-253)
  std::chrono::steady_clock::time_point cc_alg_start;
  std::chrono::steady_clock::time_point cc_alg_end;

 private:
  CCGPUSketchAlg(gs_graph* h, node_id_t V, CCAlgConfiguration cfg) : num_vertices(V), seed(0), config(cfg), g(h) {
    flush_at = 540 * get_desired_updates_per_batch();
  }

  static std::vector<Edge> to_edges(const uint32_t* e, uint64_t n) {
    std::vector<Edge> out(n);
    for (uint64_t i = 0; i < n; i++) out[i] = {e[2 * i], e[2 * i + 1]};
    return out;
  }

  struct Batches {
    std::vector<uint32_t> srcs;
    std::vector<uint64_t> starts, sizes;
    std::vector<uint32_t> dsts;
  };
  struct WorkerBuffer {
    std::mutex mtx;
    Batches q;
  };
  static constexpr int kWorkers = 256;  // thr_id is taken modulo this

  WorkerBuffer& worker(int thr_id) { return workers[(unsigned)thr_id % kWorkers]; }

  // ships batches through the C ABI; the caller holds mtx (the handle is not thread-safe)
  void ship(const Batches& b) {
    if (b.srcs.empty()) return;
    gs_throw_if(gs_ingest_vertex_batches(g, 0, b.srcs.data(), b.starts.data(), b.sizes.data(),
                                         (uint32_t)b.srcs.size(), b.dsts.data(), b.dsts.size(), 0, nullptr),
                "gs_ingest_vertex_batches");
  }

  node_id_t num_vertices;
  size_t seed;
  CCAlgConfiguration config;
  gs_graph* g = nullptr;
  std::mutex mtx;
  bool update_locked = false;
  size_t flush_at = 1;
  int num_host_threads = 1;
  std::vector<WorkerBuffer> workers = std::vector<WorkerBuffer>(kWorkers);
};

// The CPU algorithm's name maps to the same device implementation.
using CCSketchAlg = CCGPUSketchAlg;
