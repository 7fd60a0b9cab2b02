// Stand-in for StreamingUtilities' graph_zeppelin_common.h, which the reference fetches at
// configure time and does not vendor.  Only the types the reference's hot-path sources use.
// vec_hash_t is 64-bit: the reference's CUDA kernel XORs gamma with 64-bit atomics
// (src/cuda_kernel.cu:49,192), which a 32-bit type could not hold.
#pragma once
#include <cstdint>
#include <cstddef>

typedef uint32_t node_id_t;
typedef uint64_t edge_id_t;
typedef uint64_t vec_t;
typedef uint64_t vec_hash_t;

struct Edge {
  node_id_t src = 0;
  node_id_t dst = 0;
  bool operator<(const Edge& o) const { return src == o.src ? dst < o.dst : src < o.src; }
  bool operator==(const Edge& o) const { return src == o.src && dst == o.dst; }
};

enum UpdateType { INSERT = 0, DELETE = 1, BREAKPOINT = 2 };
