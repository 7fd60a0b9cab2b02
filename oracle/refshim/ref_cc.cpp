// extern "C" wrappers over the reference's own CCSketchAlg (compiled from the reference's
// sources by oracle/Makefile into oracle/_ref/libgsref.so).  TEST INFRASTRUCTURE ONLY: the
// tests use it to pin the oracle restatement, and bench.py times it as the CPU baseline.
// Built with -DNO_EAGER_DSU so that every query runs the sketch Boruvka path
// (CMakeLists.txt:104-114 documents the flag).
#include <algorithm>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "cc_sketch_alg.h"
#include "private_access.h"

static thread_local std::string g_err;

// CCSketchAlg::sketches (include/cc_sketch_alg.h:76)
struct GsCCSketches { typedef Sketch** CCSketchAlg::*type; friend type gs_ref_member(GsCCSketches); };
template struct GsRefPrivate<GsCCSketches, &CCSketchAlg::sketches>;

extern "C" {

const char* gsref_last_error() { return g_err.c_str(); }

void* gsref_cc_new(uint32_t V, uint64_t seed, double factor) {
  CCAlgConfiguration cfg;
  cfg.sketches_factor(factor);
  auto* a = new CCSketchAlg(V, seed, cfg);
  a->pre_insert({{0, 1}, INSERT}, 0);  // NO_EAGER_DSU: marks the cached DSU invalid
  return a;
}

void gsref_cc_free(void* h) { delete static_cast<CCSketchAlg*>(h); }

void gsref_cc_alloc_workers(void* h, uint32_t n) {
  static_cast<CCSketchAlg*>(h)->allocate_worker_memory(n);
}

uint64_t gsref_cc_desired_batch(void* h) {
  return static_cast<CCSketchAlg*>(h)->get_desired_updates_per_batch();
}

int gsref_cc_update(void* h, uint32_t src, uint32_t dst, int type) {
  try {
    static_cast<CCSketchAlg*>(h)->update({{src, dst}, (UpdateType)type});
  } catch (std::exception& e) { g_err = e.what(); return 1; }
  return 0;
}

// One CCSketchAlg::apply_update_batch per vertex batch, from `threads` std::threads; batch b
// goes to thread b % threads (test/cpu_sketch_throughput_stream.cpp:103-119).
int gsref_cc_ingest_batches(void* h, uint32_t threads, uint64_t num_batches, const uint32_t* srcs,
                            const uint64_t* starts, const uint64_t* sizes, const uint32_t* dsts) {
  auto* a = static_cast<CCSketchAlg*>(h);
  a->pre_insert({{0, 1}, INSERT}, 0);
  std::vector<std::thread> ts;
  std::vector<int> errs(threads, 0);
  for (uint32_t t = 0; t < threads; t++) {
    ts.emplace_back([&, t]() {
      std::vector<node_id_t> buf;
      try {
        for (uint64_t b = t; b < num_batches; b += threads) {
          buf.assign(dsts + starts[b], dsts + starts[b] + sizes[b]);
          a->apply_update_batch((int)t, srcs[b], buf);
        }
      } catch (std::exception& e) { errs[t] = 1; }
    });
  }
  for (auto& x : ts) x.join();
  for (int e : errs) if (e) { g_err = "apply_update_batch threw"; return 1; }
  return 0;
}

// labels[v] = minimum vertex id of v's component.  Returns 2 on OutOfSamplesException.
int gsref_cc_connected_components(void* h, uint32_t* labels, uint32_t* num_cc, uint32_t* rounds) {
  auto* a = static_cast<CCSketchAlg*>(h);
  try {
    a->pre_insert({{0, 1}, INSERT}, 0);
    ConnectedComponents cc = a->connected_components();
    auto sets = cc.get_component_sets();
    for (auto& s : sets) {
      uint32_t m = *s.begin();
      for (uint32_t v : s) labels[v] = m;
    }
    if (num_cc) *num_cc = (uint32_t)cc.size();
    if (rounds) *rounds = (uint32_t)a->last_query_rounds;
  } catch (OutOfSamplesException& e) { g_err = e.what(); return 2; }
  catch (std::exception& e) { g_err = e.what(); return 1; }
  return 0;
}

int gsref_cc_spanning_forest(void* h, uint32_t* edges, uint64_t* n) {
  auto* a = static_cast<CCSketchAlg*>(h);
  try {
    a->pre_insert({{0, 1}, INSERT}, 0);
    SpanningForest sf = a->calc_spanning_forest();
    const auto& es = sf.get_edges();
    for (size_t i = 0; i < es.size(); i++) { edges[2 * i] = es[i].src; edges[2 * i + 1] = es[i].dst; }
    *n = es.size();
  } catch (OutOfSamplesException& e) { g_err = e.what(); return 2; }
  catch (std::exception& e) { g_err = e.what(); return 1; }
  return 0;
}

// The bucket arrays of vertices [first, first+count) back to back (Sketch::serialize layout,
// src/sketch.cpp:204-206), straight from the reference's own Sketch objects.
int gsref_cc_sketch_bytes(void* h, uint32_t first, uint32_t count, uint8_t* out) {
  auto* a = static_cast<CCSketchAlg*>(h);
  Sketch** sk = a->*gs_ref_member(GsCCSketches());
  size_t pos = 0;
  for (uint32_t v = first; v < first + count; v++) {
    const size_t nb = sk[v]->bucket_array_bytes();
    std::memcpy(out + pos, sk[v]->get_readonly_bucket_ptr(), nb);
    pos += nb;
  }
  return 0;
}

int gsref_cc_write_binary(void* h, const char* path) {
  static_cast<CCSketchAlg*>(h)->write_binary(path);
  return 0;
}

void* gsref_cc_from_file(const char* path) {
  return CCSketchAlg::construct_from_serialized_data(path);
}

}  // extern "C"
