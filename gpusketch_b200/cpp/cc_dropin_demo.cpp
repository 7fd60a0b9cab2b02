// cc_dropin_demo.cpp - end-to-end use of the C++ drop-in classes, in the shape of the reference's
// tools/cuda_process_stream.cu:66-175: stream file -> GraphSketchDriver -> CCGPUSketchAlg ->
// connected_components().  Also exercises the per-vertex batch entry and the checkpoint.
//
//   cc_dropin_demo <stream_file> <seed> [checkpoint_out|-] [queries] [mode]
//
// mode "file" (default): the driver hands the file to the library (gs_ingest_stream_file);
// mode "generic": the driver's reader threads pull updates with get_update_buffer (any GraphStream);
// mode "batches": the reference's worker path - every record in both directions, grouped by source
//   vertex on the host into batches of get_desired_updates_per_batch() destinations (untimed, as the
//   gutters would have them ready), then apply_update_batch from 8 worker threads, flush_buffers and
//   connected_components() (timed).
// Prints "num_cc=<n> rounds=<r> label_checksum=<x>" after each of `queries` query points (the
// reference test's n/queries spacing), then "updates=<n> seconds=<t> updates_per_sec=<r>".
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "cc_gpu_sketch_alg.h"
#include "graph_sketch_driver.h"

namespace {

// A GraphStream that is not a BinaryFileStream, so the driver takes its reader-thread path.
class ForwardingStream : public GraphStream {
 public:
  explicit ForwardingStream(BinaryFileStream* s) : inner(s) {}
  node_id_t vertices() override { return inner->vertices(); }
  edge_id_t edges() override { return inner->edges(); }
  size_t get_update_buffer(GraphStreamUpdate* buf, size_t n) override { return inner->get_update_buffer(buf, n); }
  bool set_break_point(edge_id_t idx) override { return inner->set_break_point(idx); }

 private:
  BinaryFileStream* inner;
};

uint64_t label_checksum(const ConnectedComponents& cc, node_id_t V) {
  uint64_t sum = 0;
  for (node_id_t v = 0; v < V; v++) sum = sum * 1000003u + cc.labels()[v];
  return sum;
}

int run_batches(BinaryFileStream& stream, size_t seed, const char* ck) {
  const node_id_t V = stream.vertices();
  const edge_id_t n = stream.edges();
  std::vector<GraphStreamUpdate> ups(n + 1);
  size_t got = 0;
  while (got < n) {
    const size_t m = stream.get_update_buffer(ups.data() + got, n - got);
    if (m == 0 || ups[got].type == BREAKPOINT) break;
    got += m;
  }
  CCGPUSketchAlg alg(V, seed, CCAlgConfiguration().batch_factor(1));
  // group both directions of every record by source vertex (counting sort), then cut into batches
  std::vector<uint64_t> off(V + 1, 0);
  for (size_t i = 0; i < got; i++) { off[ups[i].edge.src + 1]++; off[ups[i].edge.dst + 1]++; }
  for (node_id_t v = 0; v < V; v++) off[v + 1] += off[v];
  std::vector<node_id_t> dst(off[V]);
  std::vector<uint64_t> cur(off.begin(), off.end() - 1);
  for (size_t i = 0; i < got; i++) {
    dst[cur[ups[i].edge.src]++] = ups[i].edge.dst;
    dst[cur[ups[i].edge.dst]++] = ups[i].edge.src;
  }
  const size_t bs = alg.get_desired_updates_per_batch();
  struct B { node_id_t src; std::vector<node_id_t> dsts; };
  std::vector<B> batches;
  for (node_id_t v = 0; v < V; v++)
    for (uint64_t s = off[v]; s < off[v + 1]; s += bs)
      batches.push_back({v, std::vector<node_id_t>(dst.begin() + s, dst.begin() + std::min<uint64_t>(off[v + 1], s + bs))});
  const int T = 8;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> ts;
  for (int t = 0; t < T; t++)
    ts.emplace_back([&, t]() {
      for (size_t b = t; b < batches.size(); b += T) alg.apply_update_batch(t, batches[b].src, batches[b].dsts);
    });
  for (auto& t : ts) t.join();
  alg.flush_buffers();
  ConnectedComponents cc = alg.connected_components();
  std::chrono::duration<double> dt = std::chrono::steady_clock::now() - t0;
  std::printf("num_cc=%u rounds=%zu label_checksum=%016llx\n", cc.size(), alg.last_query_rounds,
              (unsigned long long)label_checksum(cc, V));
  std::printf("updates=%llu batches=%zu seconds=%.4f updates_per_sec=%.1f\n", (unsigned long long)got,
              batches.size(), dt.count(), got / dt.count());
  if (ck && std::string(ck) != "-") alg.write_binary(ck);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s stream_file seed [checkpoint_out|-] [queries] [file|generic|batches]\n", argv[0]);
    return 2;
  }
  try {
    BinaryFileStream file(argv[1]);
    const size_t seed = std::strtoull(argv[2], nullptr, 0);
    const int queries = argc > 4 ? std::max(1, std::atoi(argv[4])) : 1;
    const std::string mode = argc > 5 ? argv[5] : "file";
    if (mode == "batches") return run_batches(file, seed, argc > 3 ? argv[3] : nullptr);
    ForwardingStream fwd(&file);
    GraphStream* stream = mode == "generic" ? static_cast<GraphStream*>(&fwd) : &file;
    CCGPUSketchAlg alg(file.vertices(), seed, CCAlgConfiguration().batch_factor(1));
    GraphSketchDriver<CCGPUSketchAlg> driver(&alg, stream, DriverConfiguration().worker_threads(4), 2);
    const edge_id_t n = file.edges();
    auto t0 = std::chrono::steady_clock::now();
    for (int q = 1; q <= queries; q++) {
      // query points as test/cc_alg_test.cpp:318-340 places them: every n / queries records, the
      // last one at the end of the stream
      const edge_id_t upto = q == queries ? END_OF_STREAM : (n / queries) * q;
      driver.process_stream_until(upto);
      driver.prep_query(CONNECTIVITY);
      alg.flush_buffers();
      ConnectedComponents cc = alg.connected_components();
      std::printf("num_cc=%u rounds=%zu label_checksum=%016llx\n", cc.size(), alg.last_query_rounds,
                  (unsigned long long)label_checksum(cc, file.vertices()));
    }
    std::chrono::duration<double> dt = std::chrono::steady_clock::now() - t0;
    std::printf("updates=%llu seconds=%.4f updates_per_sec=%.1f driver_updates=%zu\n", (unsigned long long)n,
                dt.count(), n / dt.count(), driver.get_total_updates());
    if (argc > 3 && std::string(argv[3]) != "-") alg.write_binary(argv[3]);
  } catch (std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
