// extern "C" wrappers over the reference's own MCSketchAlg (compiled from the reference's
// sources by oracle/Makefile).  TEST INFRASTRUCTURE ONLY.  Sketches are plain host Sketches
// (SketchParams::cudaUVM_enabled = false, src/mc_sketch_alg.cpp:114-119).
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "mc_sketch_alg.h"

extern "C" {

void* gsref_mc_new(uint32_t V, uint64_t seed, uint32_t num_graphs, double factor) {
  CCAlgConfiguration cfg;
  cfg.sketches_factor(factor);
  auto* a = new MCSketchAlg(V, seed, (int)num_graphs, cfg);
  SketchParams p{};
  p.cudaUVM_enabled = false;
  for (uint32_t g = 0; g < num_graphs; g++) a->create_sketch_graph((int)g, p);
  return a;
}

void gsref_mc_free(void* h) { delete static_cast<MCSketchAlg*>(h); }

void gsref_mc_update(void* h, uint32_t graph_id, uint32_t src, uint32_t dst) {
  static_cast<MCSketchAlg*>(h)->update_subgraph((int)graph_id, {{src, dst}, INSERT});
}

// k disjoint spanning forests of subgraph graph_id; forest f goes to edges + f*2*(V-1).
int gsref_mc_k_forests(void* h, uint32_t graph_id, uint32_t k, uint32_t* edges, uint64_t* sizes) {
  auto* a = static_cast<MCSketchAlg*>(h);
  try {
    auto sfs = a->calc_disjoint_spanning_forests(graph_id, k);
    size_t stride = 2 * (size_t)(a->get_num_vertices() - 1);
    for (size_t f = 0; f < sfs.size(); f++) {
      const auto& es = sfs[f].get_edges();
      for (size_t i = 0; i < es.size(); i++) {
        edges[f * stride + 2 * i] = es[i].src;
        edges[f * stride + 2 * i + 1] = es[i].dst;
      }
      sizes[f] = es.size();
    }
  } catch (OutOfSamplesException& e) { return 2; }
  catch (std::exception& e) { return 1; }
  return 0;
}

uint64_t gsref_mc_min_cut(void* h, const uint32_t* edges, uint64_t m, uint8_t* side) {
  std::vector<Edge> es(m);
  for (uint64_t i = 0; i < m; i++) es[i] = {edges[2 * i], edges[2 * i + 1]};
  MinCut mc = static_cast<MCSketchAlg*>(h)->calc_minimum_cut(es);
  if (side) for (auto v : mc.left_vertices) side[v] = 1;
  return mc.value;
}

}  // extern "C"
