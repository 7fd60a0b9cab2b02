// gpusketch_types.h - the reference's host-side value types, re-declared for the C++ drop-in
// classes over the C ABI (include/gpusketch.h).
//
// Same names and meanings as the reference: node_id_t/edge_id_t/Edge/UpdateType come from
// StreamingUtilities' graph_zeppelin_common.h, GraphUpdate from include/types.h:11-14,
// ConnectedComponents / SpanningForest from include/return_types.h, CCAlgConfiguration from
// include/cc_alg_configuration.h, the exceptions from include/cc_sketch_alg.h:25-29 and
// include/sketch.h:333-344.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <iostream>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpusketch.h"

typedef uint32_t node_id_t;
typedef uint64_t edge_id_t;
typedef uint64_t vec_t;
typedef uint64_t vec_hash_t;

// include/bucket.h:7-12: the 16-byte bucket of a vertex sketch, laid out as gs_bucket.
struct Bucket {
  vec_t alpha;
  vec_hash_t gamma;
};
static_assert(sizeof(Bucket) == sizeof(gs_bucket), "Bucket must match gs_bucket");

// The sizing functions of the reference's Sketch (include/sketch.h:63-77,196-215), which tools call to
// fill a SketchParams: num_samples = max(18, ceil(f log2 V / (1 - log2 1.2))), one column per sample,
// bkt_per_col = ceil(log2(V(V-1)/2)) + 1, bumped by one when it is a multiple of 16.  The library
// derives the same geometry from num_vertices and sketches_factor (gs_geometry_for).
class Sketch {
 public:
  static constexpr size_t default_cols_per_sample = 1;
  static vec_t calc_vector_length(node_id_t num_vertices) {
    return (vec_t)std::ceil(double(num_vertices) * (num_vertices - 1) / 2);
  }
  static size_t calc_cc_samples(node_id_t num_vertices, double f) {
    gs_geometry g{};
    if (gs_geometry_for(num_vertices, f, &g) != GS_OK) return 18;
    return g.num_samples;
  }
  static size_t calc_bkt_per_col(size_t n) {
    const size_t t = (size_t)std::ceil(std::log2((double)n)) + 1;
    return t % 16 == 0 ? t + 1 : t;
  }
};

// include/cuda_kernel.cuh:23-37: the sketch parameters the reference's tools fill and hand to
// CCGPUSketchAlg / MCGPUSketchAlg.  The library uses `seed` and derives the geometry from the vertex
// count and the configuration's sketches_factor (the same numbers the tools compute); the UVM and
// device-bucket pointers are accepted and left untouched: the sketches live in HBM owned by the library.
struct SketchParams {
  size_t num_samples = 0;
  size_t num_buckets = 0;
  size_t num_columns = 0;
  size_t bkt_per_col = 0;
  size_t seed = 0;
  bool cudaUVM_enabled = false;
  Bucket* cudaUVM_buckets = nullptr;
  Bucket* d_buckets = nullptr;
};

struct Edge {
  node_id_t src = 0;
  node_id_t dst = 0;
  bool operator<(const Edge& o) const { return src == o.src ? dst < o.dst : src < o.src; }
  bool operator==(const Edge& o) const { return src == o.src && dst == o.dst; }
};

enum UpdateType { INSERT = 0, DELETE = 1, BREAKPOINT = 2 };

struct GraphUpdate {
  Edge edge;
  UpdateType type;
};

struct GraphStreamUpdate {
  uint8_t type;
  Edge edge;
};

enum QueryCode { CONNECTIVITY = 0, KSPANNINGFORESTS = 1, MINIMUMCUT = 2 };

class UpdateLockedException : public std::exception {
 public:
  const char* what() const noexcept override {
    return "Cannot update the algorithm: Connected components currently running";
  }
};

class OutOfSamplesException : public std::runtime_error {
 public:
  explicit OutOfSamplesException(const std::string& m) : std::runtime_error(m) {}
};

// Any other non-OK status of the C ABI.
class GpuSketchException : public std::runtime_error {
 public:
  GpuSketchException(gs_status s, const std::string& where)
      : std::runtime_error(where + ": status " + std::to_string((int)s) + ": " + gs_last_error()), status(s) {}
  gs_status status;
};

inline void gs_throw_if(gs_status s, const char* where) {
  if (s == GS_OK) return;
  if (s == GS_ERR_SKETCH_FAIL) throw OutOfSamplesException(std::string(where) + ": " + gs_last_error());
  throw GpuSketchException(s, where);
}

class CCAlgConfiguration {
 public:
  CCAlgConfiguration& disk_dir(std::string d) { _disk_dir = std::move(d); return *this; }
  CCAlgConfiguration& sketches_factor(double f) {
    _sketches_factor = f > 0 ? f : 1;  // src/cc_alg_configuration.cpp:9-17
    return *this;
  }
  CCAlgConfiguration& batch_factor(double f) { _batch_factor = f > 0 ? f : 1; return *this; }
  std::string get_disk_dir() const { return _disk_dir; }
  double get_sketches_factor() const { return _sketches_factor; }
  double get_batch_factor() const { return _batch_factor; }
  friend std::ostream& operator<<(std::ostream& out, const CCAlgConfiguration& c) {
    out << "Connected Components Algorithm Configuration:\n Sketching algorithm   = CameoSketch\n"
        << " Using Eager DSU       = False\n Num sketches factor   = " << c._sketches_factor
        << "\n Batch size factor     = " << c._batch_factor << "\n On disk data location = " << c._disk_dir;
    return out;
  }

 private:
  std::string _disk_dir = ".";
  double _sketches_factor = 1;
  double _batch_factor = 1;
};

// include/return_types.h:10-24
class ConnectedComponents {
 public:
  explicit ConnectedComponents(std::vector<node_id_t> labels) : parent_arr(std::move(labels)) {
    num_cc = 0;
    for (node_id_t v = 0; v < parent_arr.size(); v++) num_cc += parent_arr[v] == v;
  }
  std::vector<std::set<node_id_t>> get_component_sets() const {
    std::map<node_id_t, std::set<node_id_t>> temp;
    for (node_id_t i = 0; i < parent_arr.size(); ++i) temp[parent_arr[i]].insert(i);
    std::vector<std::set<node_id_t>> out;
    out.reserve(temp.size());
    for (auto& kv : temp) out.push_back(std::move(kv.second));
    return out;
  }
  bool is_connected(node_id_t a, node_id_t b) const { return parent_arr[a] == parent_arr[b]; }
  node_id_t size() const { return num_cc; }
  const std::vector<node_id_t>& labels() const { return parent_arr; }

 private:
  std::vector<node_id_t> parent_arr;
  node_id_t num_cc;
};

// include/return_types.h:26-38
class SpanningForest {
 public:
  SpanningForest() = default;
  explicit SpanningForest(std::vector<Edge> e) : edges(std::move(e)) {}
  const std::vector<Edge>& get_edges() const { return edges; }
  const std::vector<Edge>& get_sorted_adjacency() {
    if (has_adjacency) return sorted_adjacency;
    sorted_adjacency.clear();
    for (const Edge& e : edges) {
      sorted_adjacency.push_back(e);
      sorted_adjacency.push_back({e.dst, e.src});
    }
    std::sort(sorted_adjacency.begin(), sorted_adjacency.end());
    has_adjacency = true;
    return sorted_adjacency;
  }

 private:
  std::vector<Edge> edges;
  std::vector<Edge> sorted_adjacency;
  bool has_adjacency = false;
};

struct MinCut {
  std::set<node_id_t> left_vertices;
  std::set<node_id_t> right_vertices;
  size_t value;
};
