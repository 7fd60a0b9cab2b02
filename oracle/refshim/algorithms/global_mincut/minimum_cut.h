// Stand-in for VieCut's minimum_cut interface.  perform_minimum_cut computes the exact
// global minimum cut with the oracle's Stoer-Wagner (small test graphs only) and marks
// one side with setNodeInCut, which is what MCSketchAlg::calc_minimum_cut reads back.
#pragma once
#include <cstdint>
#include <memory>
#include <vector>
#include "../../data_structure/mutable_graph.h"

extern "C" uint64_t or_stoer_wagner(uint32_t V, const uint32_t* edges, uint64_t m, uint8_t* side);

namespace VieCut {
class minimum_cut {
 public:
  virtual ~minimum_cut() {}
  virtual EdgeWeight perform_minimum_cut(std::shared_ptr<mutable_graph> G) = 0;
};

template <class GraphPtr>
class viecut : public minimum_cut {
 public:
  EdgeWeight perform_minimum_cut(std::shared_ptr<mutable_graph> G) override {
    std::vector<uint8_t> side(G->n);
    uint64_t v = or_stoer_wagner(G->n, G->edges.data(), G->edges.size() / 2, side.data());
    for (uint32_t i = 0; i < G->n; i++) G->in_cut[i] = side[i];
    return (EdgeWeight)v;
  }
};
}  // namespace VieCut
