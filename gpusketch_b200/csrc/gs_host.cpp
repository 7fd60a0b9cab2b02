// gs_host.cpp - host-side pieces of the library: sketch geometry, error slot, tuning table and
// the Erdos-Renyi stream generator.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "gs_internal.h"

static thread_local std::string g_last_error;

void gs_set_error(const std::string& msg) { g_last_error = msg; }

extern "C" const char* gs_last_error(void) { return g_last_error.c_str(); }

// Sketch::calc_vector_length / calc_cc_samples / calc_bkt_per_col (include/sketch.h:177-191,312-320)
// and the Sketch constructor's column and bucket counts (src/sketch.cpp:24-30); the double
// arithmetic is the reference's, so the sizes match it for every V.
GsGeom gs_make_geom(uint32_t V, double f) {
  GsGeom g{};
  g.V = V;
  const double vec_len_d = std::ceil(double(V) * (double(V) - 1) / 2);
  const uint64_t vec_len = (uint64_t)vec_len_d;
  size_t samples = (size_t)std::ceil(f * std::log2((double)V) / (1 - 0.263034406));
  samples = std::max<size_t>(18, samples);
  size_t bkt = (size_t)(std::ceil(std::log2((double)vec_len)) + 1);
  if (bkt % 16 == 0) bkt += 1;
  g.num_samples = (uint32_t)samples;
  g.num_columns = (uint32_t)samples;  // cols_per_sample = 1 (CameoSketch)
  g.bkt_per_col = (uint32_t)bkt;
  g.num_buckets = (uint32_t)(samples * bkt + 1);
  return g;
}

extern "C" gs_status gs_geometry_for(uint32_t num_vertices, double sketches_factor, gs_geometry* out) {
  if (!out || num_vertices < 2) {
    gs_set_error("gs_geometry_for: need num_vertices >= 2 and a non-null output");
    return GS_ERR_BAD_ARG;
  }
  if (!(sketches_factor > 0)) sketches_factor = 1;
  GsGeom g = gs_make_geom(num_vertices, sketches_factor);
  out->num_vertices = num_vertices;
  out->num_samples = g.num_samples;
  out->cols_per_sample = 1;
  out->num_columns = g.num_columns;
  out->bkt_per_col = g.bkt_per_col;
  out->num_buckets = g.num_buckets;
  out->bytes_per_vertex = (uint64_t)g.num_buckets * sizeof(GsBucket);
  return GS_OK;
}

extern "C" uint64_t gs_hash64(uint64_t key, uint64_t seed) { return gs_xxh3_8(key, seed); }

GsTuning gs_tune_for(const GsGeom& geom, int num_sms) {
  (void)num_sms;
  GsTuning t;
  t.chunk = 1024;          // defaults measured best on B200 for the V=2^17 R-MAT stream; the
  t.warps_per_block = 16;  // autotuner refines them per geometry
  t.reg_depth = 0;         // every depth < 10 in the lane's shared-memory rows (fewest instructions)
  return t;
}

// ---------------------------------------------------------------------------------------
// Erdos-Renyi dynamic stream: G(V, p) edges (pairs i<j kept with probability p, found by
// geometric skipping), inserted in Fisher-Yates order, then a delete_frac share of them deleted
// and a reinsert_frac share of the deleted ones inserted again.
// ---------------------------------------------------------------------------------------
namespace {
struct SplitMix {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};
}  // namespace

extern "C" gs_status gs_gen_er_stream(uint32_t V, double p, uint64_t seed, double delete_frac,
                                      double reinsert_frac, uint32_t* pairs, uint64_t capacity, uint64_t* n) {
  if (V < 2 || !(p >= 0 && p <= 1) || !n) {
    gs_set_error("gs_gen_er_stream: bad arguments");
    return GS_ERR_BAD_ARG;
  }
  SplitMix rng{seed};
  std::vector<uint64_t> edges;
  const uint64_t total_pairs = (uint64_t)V * (V - 1) / 2;
  if (p > 0) {
    // pair index k enumerates (i, j), i < j, row by row
    const double lq = std::log1p(-std::min(p, 1.0 - 1e-16));
    uint64_t k = 0;
    uint32_t i = 0;
    uint64_t row_start = 0;  // index of (i, i+1)
    for (;;) {
      if (p < 1) {
        double u = rng.uniform();
        if (u <= 0) u = 1e-300;
        const double skip = std::floor(std::log(u) / lq);
        if (skip >= (double)(total_pairs - k)) break;
        k += (uint64_t)skip;
      }
      if (k >= total_pairs) break;
      while (k >= row_start + (V - 1 - i)) { row_start += V - 1 - i; i++; }
      const uint32_t j = (uint32_t)(i + 1 + (k - row_start));
      edges.push_back(((uint64_t)i << 32) | j);
      k++;
    }
  }
  for (uint64_t t = edges.size(); t > 1; t--) std::swap(edges[t - 1], edges[rng.below(t)]);
  const uint64_t m = edges.size();
  std::vector<uint64_t> order(m);
  for (uint64_t t = 0; t < m; t++) order[t] = t;
  for (uint64_t t = m; t > 1; t--) std::swap(order[t - 1], order[rng.below(t)]);
  const uint64_t ndel = (uint64_t)std::floor(delete_frac * (double)m);
  std::vector<uint64_t> dels(order.begin(), order.begin() + std::min(ndel, m));
  for (uint64_t t = dels.size(); t > 1; t--) std::swap(dels[t - 1], dels[rng.below(t)]);
  const uint64_t nre = (uint64_t)std::floor(reinsert_frac * (double)dels.size());
  const uint64_t total = m + dels.size() + nre;
  *n = total;
  if (!pairs) return GS_OK;
  if (capacity < total) {
    gs_set_error("gs_gen_er_stream: capacity " + std::to_string(capacity) + " < " + std::to_string(total));
    return GS_ERR_BAD_ARG;
  }
  uint64_t w = 0;
  auto put = [&](uint64_t e) { pairs[2 * w] = (uint32_t)(e >> 32); pairs[2 * w + 1] = (uint32_t)e; w++; };
  for (uint64_t t = 0; t < m; t++) put(edges[t]);
  for (uint64_t t = 0; t < dels.size(); t++) put(edges[dels[t]]);
  for (uint64_t t = 0; t < nre; t++) put(edges[dels[t]]);
  return GS_OK;
}
