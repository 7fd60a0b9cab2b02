// mc_gpu_sketch_alg.h - MCGPUSketchAlg drop-in: k-connectivity / minimum cut over sketch subgraphs
// (include/mc_sketch_alg.h:73-304, include/mc_gpu_sketch_alg.h:118-273) on the C ABI.
//
// Every edge record is tagged on the device with level = get_index_depth(e, seed, num_subgraphs-1)
// (src/mc_gpu_sketch_alg.cpp:160) and toggled in levels 0..min(level, max_sketch_graphs-1).
#pragma once

#include <cmath>
#include <mutex>
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

  int get_num_sketch_graphs() { return (int)levels; }

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
