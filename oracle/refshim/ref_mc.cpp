// extern "C" wrappers over the reference's own MCSketchAlg (compiled from the reference's
// sources by oracle/Makefile).  TEST INFRASTRUCTURE ONLY.  Sketches are plain host Sketches
// (SketchParams::cudaUVM_enabled = false, src/mc_sketch_alg.cpp:114-119).
#include <algorithm>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "mc_sketch_alg.h"
#include "private_access.h"

// MCSketchAlg::sketches (include/mc_sketch_alg.h:86): graph g's vertex v at [g*V + v]
struct GsMCSketches { typedef Sketch** MCSketchAlg::*type; friend type gs_ref_member(GsMCSketches); };
template struct GsRefPrivate<GsMCSketches, &MCSketchAlg::sketches>;

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

// The reference GPU driver's subgraph fan-out, on the host: record (src, dst) gets the tag
// get_index_depth(concat_pairing_fn(src, dst), seed, num_subgraphs - 1) and is inserted into sketch
// graphs 0 .. min(tag, num_graphs - 1) (MCGPUSketchAlg::apply_update_batch and
// complete_update_batch, src/mc_gpu_sketch_alg.cpp:139-178,83-137; every subgraph stays sketched).
void gsref_mc_ingest_tagged(void* h, const uint32_t* pairs, uint64_t n, uint32_t num_subgraphs,
                            uint32_t num_graphs) {
  auto* a = static_cast<MCSketchAlg*>(h);
  const size_t seed = a->get_seed();
  for (uint64_t i = 0; i < n; i++) {
    const node_id_t u = pairs[2 * i], v = pairs[2 * i + 1];
    const vec_t e = static_cast<vec_t>(concat_pairing_fn(u, v));
    const size_t tag = Bucket_Boruvka::get_index_depth(e, seed, num_subgraphs - 1);
    const size_t top = std::min<size_t>(tag, num_graphs - 1);
    for (size_t g = 0; g <= top; g++) a->update_subgraph((int)g, {{u, v}, INSERT});
  }
}

// Sketch bytes of graph g, vertices 0..V-1 back to back (Sketch::serialize layout).
int gsref_mc_level_bytes(void* h, uint32_t graph_id, uint8_t* out) {
  auto* a = static_cast<MCSketchAlg*>(h);
  Sketch** sk = a->*gs_ref_member(GsMCSketches());
  const node_id_t V = a->get_num_vertices();
  size_t pos = 0;
  for (node_id_t v = 0; v < V; v++) {
    const Sketch* s = sk[(size_t)graph_id * V + v];
    std::memcpy(out + pos, s->get_readonly_bucket_ptr(), s->bucket_array_bytes());
    pos += s->bucket_array_bytes();
  }
  return 0;
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
