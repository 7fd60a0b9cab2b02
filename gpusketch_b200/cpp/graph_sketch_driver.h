// graph_sketch_driver.h - GraphSketchDriver drop-in and the binary stream reader.
//
// The reference driver (include/graph_sketch_driver.h:70-232) pushes every stream update into a
// guttering system on the host, and worker threads hand per-vertex batches to
// Alg::apply_update_batch.  Here the grouping by endpoint happens on the device, so reader threads
// gather raw (src, dst) records and hand them in bulk to Alg::ingest_records; batch_callback keeps
// the reference's per-vertex entry for callers that already hold vertex batches.
//
// BinaryFileStream reads the StreamingUtilities binary stream format used by the reference's
// tools and tests (test/res/multiples_graph_1024_stream.data): a header {u32 num_vertices,
// u64 num_updates} followed by packed 9-byte records {u8 type (0 insert, 1 delete), u32 src,
// u32 dst}.
#pragma once

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gpusketch_types.h"

constexpr edge_id_t END_OF_STREAM = (edge_id_t)-1;

class GraphStream {
 public:
  virtual ~GraphStream() = default;
  virtual node_id_t vertices() = 0;
  virtual edge_id_t edges() = 0;
  // fills up to `n` updates; a BREAKPOINT update marks the break point / end of the stream
  virtual size_t get_update_buffer(GraphStreamUpdate* buf, size_t n) = 0;
  virtual bool set_break_point(edge_id_t idx) = 0;
  virtual bool get_update_is_thread_safe() { return true; }
};

class BinaryFileStream : public GraphStream {
 public:
  explicit BinaryFileStream(const std::string& path) {
    f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open stream file " + path);
    uint8_t hdr[12];
    if (std::fread(hdr, 1, 12, f) != 12) throw std::runtime_error("truncated stream header in " + path);
    std::memcpy(&num_vertices, hdr, 4);
    std::memcpy(&num_updates, hdr + 4, 8);
    break_idx = num_updates;
  }
  ~BinaryFileStream() override {
    if (f) std::fclose(f);
  }
  node_id_t vertices() override { return num_vertices; }
  edge_id_t edges() override { return num_updates; }

  bool set_break_point(edge_id_t idx) override {
    std::lock_guard<std::mutex> lk(mtx);
    if (idx != END_OF_STREAM && idx < next) return false;
    break_idx = idx == END_OF_STREAM ? num_updates : std::min<edge_id_t>(idx, num_updates);
    return true;
  }

  size_t get_update_buffer(GraphStreamUpdate* buf, size_t n) override {
    std::lock_guard<std::mutex> lk(mtx);
    if (n == 0) return 0;
    const edge_id_t left = break_idx - next;
    if (left == 0) {
      buf[0].type = BREAKPOINT;
      buf[0].edge = {0, 0};
      return 1;
    }
    const size_t m = (size_t)std::min<edge_id_t>(left, n);
    raw.resize(m * 9);
    if (std::fseek(f, (long)(12 + next * 9), SEEK_SET) != 0 || std::fread(raw.data(), 9, m, f) != m)
      throw std::runtime_error("stream file read failed");
    for (size_t i = 0; i < m; i++) {
      buf[i].type = raw[9 * i];
      std::memcpy(&buf[i].edge.src, &raw[9 * i + 1], 4);
      std::memcpy(&buf[i].edge.dst, &raw[9 * i + 5], 4);
    }
    next += m;
    return m;
  }

  // writes a stream file in the same format (test and tool helper)
  static void write(const std::string& path, node_id_t V, const std::vector<GraphStreamUpdate>& ups) {
    FILE* o = std::fopen(path.c_str(), "wb");
    if (!o) throw std::runtime_error("cannot create " + path);
    uint64_t n = ups.size();
    std::fwrite(&V, 4, 1, o);
    std::fwrite(&n, 8, 1, o);
    for (const auto& u : ups) {
      std::fwrite(&u.type, 1, 1, o);
      std::fwrite(&u.edge.src, 4, 1, o);
      std::fwrite(&u.edge.dst, 4, 1, o);
    }
    std::fclose(o);
  }

 private:
  FILE* f = nullptr;
  node_id_t num_vertices = 0;
  edge_id_t num_updates = 0;
  edge_id_t next = 0;
  edge_id_t break_idx = 0;
  std::mutex mtx;
  std::vector<uint8_t> raw;
};

enum GutterSystem { GUTTERTREE, STANDALONE, CACHETREE };

// include/driver_configuration.h:12-48.  The gutter choice is accepted for source compatibility;
// records are grouped by endpoint on the device whatever it says.
class DriverConfiguration {
 public:
  DriverConfiguration& gutter_sys(GutterSystem s) { _gutter_sys = s; return *this; }
  DriverConfiguration& disk_dir(std::string d) { _disk_dir = std::move(d); return *this; }
  DriverConfiguration& worker_threads(size_t n) { _num_worker_threads = n ? n : 1; return *this; }
  GutterSystem get_gutter_sys() const { return _gutter_sys; }
  std::string get_disk_dir() const { return _disk_dir; }
  size_t get_worker_threads() const { return _num_worker_threads; }

 private:
  GutterSystem _gutter_sys = STANDALONE;
  std::string _disk_dir = ".";
  size_t _num_worker_threads = 1;
};

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
