// Stand-in for VieCut's mutable_graph: stores the edge list handed to calc_minimum_cut.
#pragma once
#include <cstdint>
#include <vector>

namespace VieCut {
typedef uint64_t EdgeWeight;
class mutable_graph {
 public:
  uint32_t n = 0;
  std::vector<uint32_t> edges;
  std::vector<uint8_t> in_cut;
  void start_construction(uint32_t nodes, uint64_t m) {
    n = nodes; edges.clear(); edges.reserve(2 * m); in_cut.assign(nodes, 0);
  }
  void new_edge(uint32_t a, uint32_t b) { edges.push_back(a); edges.push_back(b); }
  void finish_construction() {}
  void computeDegrees() {}
  bool getNodeInCut(uint32_t i) const { return in_cut[i] != 0; }
};
}  // namespace VieCut
