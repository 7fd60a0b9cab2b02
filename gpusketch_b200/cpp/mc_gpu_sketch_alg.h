// mc_gpu_sketch_alg.h - MCGPUSketchAlg drop-in: k-connectivity / minimum cut over sketch subgraphs
// (include/mc_sketch_alg.h:73-304, include/mc_gpu_sketch_alg.h:118-273) on the C ABI.
//
// Every edge record is tagged on the device with level = get_index_depth(e, seed, num_subgraphs-1)
// (src/mc_gpu_sketch_alg.cpp:160) and toggled in levels 0..min(level, max_sketch_graphs-1).
#pragma once

#include <algorithm>
#include <cmath>
#include <iostream>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpusketch_types.h"

class MCGPUSketchAlg {
 public:
  MCGPUSketchAlg(node_id_t num_vertices, size_t seed, int num_subgraphs, int max_sketch_graphs, int k,
                 CCAlgConfiguration config = CCAlgConfiguration(), int device = -1)
      : num_vertices(num_vertices), seed(seed), k(k), levels((uint32_t)max_sketch_graphs), config(config) {
    gs_graph_config cfg{};
    cfg.num_vertices = num_vertices;
    cfg.num_levels = (uint32_t)max_sketch_graphs;
    cfg.num_subgraphs = (uint32_t)num_subgraphs;
    cfg.seed = seed;
    cfg.sketches_factor = config.get_sketches_factor();
    cfg.batch_factor = config.get_batch_factor();
    cfg.device = device;
    gs_throw_if(gs_graph_create(&cfg, &g), "gs_graph_create");
  }
  // The reference's constructor (include/mc_gpu_sketch_alg.h:168-230, called by tools/min_cut.cu:169):
  // max_sketch_graphs sketch levels of the geometry num_vertices and config.sketches_factor give (the
  // tool sets that factor to its reduced_k), tags bounded by num_subgraphs, the sketch seed from the
  // SketchParams, and the adaptive exact tier of the reference's EdgeStore: initial_sketch_graphs
  // levels sketched at the start, one more whenever the stored edges outgrow sketch_bytes.  k is the
  // number of forests per level the level loop (min_cut()) takes; num_threads worker threads and
  // num_reader_threads readers only sized the reference's host buffers.
  MCGPUSketchAlg(node_id_t num_vertices, int num_threads, int num_reader_threads, SketchParams sketch_params,
                 int num_subgraphs, int max_sketch_graphs, int k, size_t sketch_bytes, int initial_sketch_graphs,
                 CCAlgConfiguration config)
      : MCGPUSketchAlg(num_vertices, sketch_params.seed, num_subgraphs, std::max(1, max_sketch_graphs), k, config) {
    (void)num_threads;
    (void)num_reader_threads;
    if (initial_sketch_graphs > max_sketch_graphs)
      throw std::invalid_argument("initial sketch graphs exceed the maximum number of sketch graphs");
    // with max_sketch_graphs 0 the reference keeps every edge exactly and has no level to contract into
    // (its contraction would index past its subgraph array); here one level stays available for that
    gs_throw_if(gs_graph_set_edge_store(g, (uint32_t)std::max(0, initial_sketch_graphs), sketch_bytes),
                "gs_graph_set_edge_store");
  }

  ~MCGPUSketchAlg() { gs_graph_destroy(g); }
  MCGPUSketchAlg(const MCGPUSketchAlg&) = delete;
  MCGPUSketchAlg& operator=(const MCGPUSketchAlg&) = delete;

  // driver contract
  void allocate_worker_memory(size_t) {}
  size_t get_desired_updates_per_batch() { return gs_desired_updates_per_batch(g); }
  node_id_t get_num_vertices() { return num_vertices; }
  void pre_insert(GraphUpdate, int = 0) {}
  bool has_cached_query(int) { return false; }
  void print_configuration() { std::cout << config << std::endl; }

  void ingest_records(const uint32_t* pairs, size_t n) {
    std::lock_guard<std::mutex> lk(mtx);
    gs_throw_if(gs_ingest_pairs(g, pairs, n, 0, nullptr), "gs_ingest_pairs");
  }
  void update(GraphUpdate upd) {
    uint32_t p[2] = {upd.edge.src, upd.edge.dst};
    ingest_records(p, 1);
  }
  // MCGPUSketchAlg::apply_flush_updates (src/mc_gpu_sketch_alg.cpp:180-205)
  void apply_flush_updates() { gs_throw_if(gs_synchronize(g), "gs_synchronize"); }

  // levels sketched now: the initial ones plus one per contraction of the exact tier
  int get_num_sketch_graphs() {
    uint32_t lv = 0;
    gs_throw_if(gs_graph_sketched_levels(g, &lv, nullptr), "gs_graph_sketched_levels");
    return (int)lv;
  }

  // the exact tier's edges (MCGPUSketchAlg::get_adjlist_spanning_forests, src/mc_gpu_sketch_alg.cpp:207-209):
  // every present edge whose tag passes the sketched levels
  std::vector<Edge> get_adjlist_spanning_forests() {
    gs_throw_if(gs_synchronize(g), "gs_synchronize");
    uint32_t lv = 0;
    gs_throw_if(gs_graph_sketched_levels(g, &lv, nullptr), "gs_graph_sketched_levels");
    uint64_t n = 0;
    gs_throw_if(gs_edge_store_edges(g, lv, nullptr, 0, &n), "gs_edge_store_edges");
    std::vector<uint32_t> e(2 * n + 2);
    gs_throw_if(gs_edge_store_edges(g, lv, e.data(), n, &n), "gs_edge_store_edges");
    std::vector<Edge> out(n);
    for (uint64_t i = 0; i < n; i++) out[i] = {e[2 * i], e[2 * i + 1]};
    return out;
  }

  // MCGPUSketchAlg::print_subgraph_edges (include/mc_gpu_sketch_alg.h:253-260)
  void print_subgraph_edges() {
    uint32_t lv = 0;
    uint64_t contractions = 0, n = 0;
    gs_throw_if(gs_graph_sketched_levels(g, &lv, &contractions), "gs_graph_sketched_levels");
    gs_throw_if(gs_edge_store_edges(g, lv, nullptr, 0, &n), "gs_edge_store_edges");
    std::cout << "Sketch subgraphs: " << lv << " (" << contractions << " contractions of the exact tier)\n";
    std::cout << "  Adjacency list:      " << n << std::endl;
  }

  void display_time() {
    gs_profile p{};
    gs_throw_if(gs_profile_read(g, &p), "gs_profile_read");
    std::cout << "Device ingest: " << p.records_ingested << " edge records, " << p.kernel_launches
              << " kernel launches\n";
  }

  // records [first, first+count) of a binary stream file, read by the library (gs_ingest_stream_file)
  void ingest_stream_file(const std::string& path, edge_id_t first, edge_id_t count) {
    std::lock_guard<std::mutex> lk(mtx);
    gs_throw_if(gs_ingest_stream_file(g, path.c_str(), first, count, nullptr), "gs_ingest_stream_file");
  }

  // MCSketchAlg::calc_disjoint_spanning_forests (src/mc_sketch_alg.cpp:889-919)
  std::vector<SpanningForest> calc_disjoint_spanning_forests(size_t graph_id, size_t kk) {
    const size_t stride = 2 * (size_t)(num_vertices - 1);
    std::vector<uint32_t> e(kk * stride);
    std::vector<uint64_t> sizes(kk);
    gs_throw_if(gs_disjoint_spanning_forests(g, (uint32_t)graph_id, (uint32_t)kk, e.data(), sizes.data()),
                "gs_disjoint_spanning_forests");
    std::vector<SpanningForest> out;
    for (size_t f = 0; f < kk; f++) {
      std::vector<Edge> es(sizes[f]);
      for (uint64_t i = 0; i < sizes[f]; i++) es[i] = {e[f * stride + 2 * i], e[f * stride + 2 * i + 1]};
      out.emplace_back(std::move(es));
    }
    return out;
  }

  // MCSketchAlg::calc_minimum_cut (src/mc_sketch_alg.cpp:966-1002) with the library's exact min cut
  MinCut calc_minimum_cut(const std::vector<Edge>& edges) {
    std::vector<uint32_t> p(2 * edges.size());
    for (size_t i = 0; i < edges.size(); i++) { p[2 * i] = edges[i].src; p[2 * i + 1] = edges[i].dst; }
    uint64_t v = 0;
    std::vector<uint8_t> side(num_vertices);
    gs_throw_if(gs_exact_min_cut(num_vertices, p.data(), edges.size(), &v, side.data()), "gs_exact_min_cut");
    MinCut mc;
    for (node_id_t i = 0; i < num_vertices; i++) (side[i] ? mc.left_vertices : mc.right_vertices).insert(i);
    mc.value = v;
    return mc;
  }

  // the level loop of tools/min_cut.cu:208-252: value * 2^level at the first level whose cut < k
  size_t min_cut(uint32_t* level_found = nullptr) {
    uint64_t value = 0, cut = 0;
    uint32_t lvl = 0;
    gs_throw_if(gs_min_cut(g, (uint32_t)k, &value, &lvl, &cut, nullptr), "gs_min_cut");
    if (level_found) *level_found = lvl;
    return value;
  }

  gs_graph* handle() { return g; }

 private:
  node_id_t num_vertices;
  size_t seed;
  int k;
  uint32_t levels;
  CCAlgConfiguration config;
  gs_graph* g = nullptr;
  std::mutex mtx;
};
