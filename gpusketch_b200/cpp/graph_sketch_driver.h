// graph_sketch_driver.h - GraphSketchDriver drop-in.
//
// The reference driver (include/graph_sketch_driver.h:70-232) pushes every stream update into a
// guttering system on the host, and worker threads hand per-vertex batches to
// Alg::apply_update_batch.  Here the grouping by endpoint happens on the device:
//   * a BinaryFileStream whose algorithm can ingest a file range (Alg::ingest_stream_file) is read by
//     the library itself (gs_ingest_stream_file: file -> page-locked ring -> device decode and
//     bucketing), with no per-update host work;
//   * any other stream is read by the reader threads, which gather raw (src, dst) records and hand
//     them in bulk to Alg::ingest_records.
// batch_callback keeps the reference's per-vertex entry for callers that already hold vertex batches.
#pragma once

#include <unistd.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

#include "binary_file_stream.h"
#include "gpusketch_types.h"

enum GutterSystem { GUTTERTREE, STANDALONE, CACHETREE };

// The guttering system's settings (GutterTree's GutteringConfiguration, used by the reference's tools,
// tools/cuda_process_stream.cu:121).  Accepted for source compatibility: records are grouped by endpoint
// on the device, so there are no host gutters to configure.
class GutteringConfiguration {
 public:
  GutteringConfiguration& page_factor(int) { return *this; }
  GutteringConfiguration& buffer_exp(int) { return *this; }
  GutteringConfiguration& fanout(int) { return *this; }
  GutteringConfiguration& num_flushers(int) { return *this; }
  GutteringConfiguration& gutter_factor(float) { return *this; }
  GutteringConfiguration& queue_factor(int) { return *this; }
  GutteringConfiguration& wq_batch_per_elm(int) { return *this; }
};

// include/driver_configuration.h:12-48.  The gutter choice is accepted for source compatibility;
// records are grouped by endpoint on the device whatever it says.
class DriverConfiguration {
 public:
  DriverConfiguration& gutter_sys(GutterSystem s) { _gutter_sys = s; return *this; }
  DriverConfiguration& disk_dir(std::string d) { _disk_dir = std::move(d); return *this; }
  DriverConfiguration& worker_threads(size_t n) { _num_worker_threads = n ? n : 1; return *this; }
  GutteringConfiguration& gutter_conf() { return _gutter_conf; }
  GutterSystem get_gutter_sys() const { return _gutter_sys; }
  std::string get_disk_dir() const { return _disk_dir; }
  size_t get_worker_threads() const { return _num_worker_threads; }

 private:
  GutterSystem _gutter_sys = STANDALONE;
  std::string _disk_dir = ".";
  size_t _num_worker_threads = 1;
  GutteringConfiguration _gutter_conf;
};

// Alg::ingest_stream_file(path, first, count) exists
template <class Alg, class = void>
struct GsIngestsFiles : std::false_type {};
template <class Alg>
struct GsIngestsFiles<Alg, std::void_t<decltype(std::declval<Alg&>().ingest_stream_file(
                               std::declval<const std::string&>(), edge_id_t(), edge_id_t()))>> : std::true_type {};

template <class Alg>
class GraphSketchDriver {
 public:
  GraphSketchDriver(Alg* sketching_alg, GraphStream* stream, DriverConfiguration config,
                    size_t num_stream_threads = 1)
      : alg(sketching_alg), stream(stream), num_stream_threads(num_stream_threads ? num_stream_threads : 1) {
    alg->allocate_worker_memory(config.get_worker_threads());
    if (this->num_stream_threads > 1 && !stream->get_update_is_thread_safe()) this->num_stream_threads = 1;
    total_updates = 0;
  }

  // include/graph_sketch_driver.h:141-191: all updates before break_edge_idx are applied
  void process_stream_until(edge_id_t break_edge_idx) {
    if (!stream->set_break_point(break_edge_idx))
      throw std::runtime_error("Could not correctly set breakpoint: " + std::to_string(break_edge_idx));
    if constexpr (GsIngestsFiles<Alg>::value) {
      if (auto* file = dynamic_cast<BinaryFileStream*>(stream)) {
        edge_id_t first = 0, n = 0;
        if (file->claim(&first, &n)) {
          alg->ingest_stream_file(file->path(), first, n);
          total_updates += 2 * n;
        }
        return;
      }
    }
    auto task = [&]() {
      std::vector<GraphStreamUpdate> buf(update_array_size);
      std::vector<uint32_t> pairs;
      pairs.reserve(2 * ship_records);
      for (;;) {
        const size_t got = stream->get_update_buffer(buf.data(), buf.size());
        bool done = false;
        for (size_t i = 0; i < got; i++) {
          if (buf[i].type == BREAKPOINT) { done = true; break; }
          alg->pre_insert({buf[i].edge, (UpdateType)buf[i].type}, 0);
          pairs.push_back(buf[i].edge.src);
          pairs.push_back(buf[i].edge.dst);
        }
        if (pairs.size() >= 2 * ship_records || (done && !pairs.empty())) {
          total_updates += 2 * (pairs.size() / 2);
          alg->ingest_records(pairs.data(), pairs.size() / 2);
          pairs.clear();
        }
        if (done || got == 0) return;
      }
    };
    std::vector<std::thread> ts;
    for (size_t i = 0; i < num_stream_threads; i++) ts.emplace_back(task);
    for (auto& t : ts) t.join();
  }

  // include/graph_sketch_driver.h:193-202: the records are already on the device
  void prep_query(int query_code) { (void)query_code; }

  // include/graph_sketch_driver.h:204-208
  void batch_callback(int thr_id, node_id_t src_vertex, const std::vector<node_id_t>& dst_vertices) {
    total_updates += dst_vertices.size();
    alg->apply_update_batch(thr_id, src_vertex, dst_vertices);
  }

  size_t get_total_updates() { return total_updates.load(); }

 private:
  static constexpr size_t update_array_size = 4096;
  static constexpr size_t ship_records = 1 << 22;
  Alg* alg;
  GraphStream* stream;
  size_t num_stream_threads;
  std::atomic<size_t> total_updates;
};
