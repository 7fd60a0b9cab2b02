// binary_file_stream.h - the graph-stream interface of the driver and the binary stream file reader.
//
// BinaryFileStream reads the StreamingUtilities binary stream format used by the reference's tools
// and tests (test/res/multiples_graph_1024_stream.data): a header {u32 num_vertices,
// u64 num_updates} followed by packed 9-byte records {u8 type (0 insert, 1 delete), u32 src,
// u32 dst}.  get_update_buffer hands out updates one buffer at a time, as the reference's reader
// threads take them; claim() hands a whole record range to a caller that ingests it straight from the
// file (GraphSketchDriver does so through gs_ingest_stream_file, which reads the file into the
// library's page-locked ring and decodes the records on the device).
#pragma once

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
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
  explicit BinaryFileStream(const std::string& path) : file_path(path) {
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

  // Hands records [*first, *first + *n) up to the break point to the caller, who reads them from the
  // file itself; false when none are left before the break point.
  bool claim(edge_id_t* first, edge_id_t* n) {
    std::lock_guard<std::mutex> lk(mtx);
    if (next >= break_idx) return false;
    *first = next;
    *n = break_idx - next;
    next = break_idx;
    return true;
  }
  const std::string& path() const { return file_path; }

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
  std::string file_path;
  FILE* f = nullptr;
  node_id_t num_vertices = 0;
  edge_id_t num_updates = 0;
  edge_id_t next = 0;
  edge_id_t break_idx = 0;
  std::mutex mtx;
  std::vector<uint8_t> raw;
};
