// cc_dropin_demo.cpp - end-to-end use of the C++ drop-in classes, in the shape of the reference's
// tools/cuda_process_stream.cu:66-175: stream file -> GraphSketchDriver -> CCGPUSketchAlg ->
// connected_components().  Also exercises the per-vertex batch entry and the checkpoint.
//
//   cc_dropin_demo <stream_file> <seed> [checkpoint_out] [queries]
// prints "num_cc=<n> rounds=<r> label_checksum=<x>" after each of `queries` evenly spaced queries.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "cc_gpu_sketch_alg.h"
#include "graph_sketch_driver.h"

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s stream_file seed [checkpoint_out] [queries]\n", argv[0]);
    return 2;
  }
  try {
    BinaryFileStream stream(argv[1]);
    const size_t seed = std::strtoull(argv[2], nullptr, 0);
    const int queries = argc > 4 ? std::atoi(argv[4]) : 1;
    CCGPUSketchAlg alg(stream.vertices(), seed, CCAlgConfiguration().batch_factor(1));
    GraphSketchDriver<CCGPUSketchAlg> driver(&alg, &stream, DriverConfiguration().worker_threads(4), 2);
    const edge_id_t n = stream.edges();
    auto t0 = std::chrono::steady_clock::now();
    for (int q = 1; q <= queries; q++) {
      // query points as test/cc_alg_test.cpp:318-340 places them: every n / queries records, the
      // last one at the end of the stream
      const edge_id_t upto = q == queries ? END_OF_STREAM : (n / queries) * q;
      driver.process_stream_until(upto);
      driver.prep_query(CONNECTIVITY);
      alg.flush_buffers();
      ConnectedComponents cc = alg.connected_components();
      uint64_t sum = 0;
      for (node_id_t v = 0; v < stream.vertices(); v++) sum = sum * 1000003u + cc.labels()[v];
      std::printf("num_cc=%u rounds=%zu label_checksum=%016llx\n", cc.size(), alg.last_query_rounds,
                  (unsigned long long)sum);
    }
    std::chrono::duration<double> dt = std::chrono::steady_clock::now() - t0;
    std::printf("updates=%llu seconds=%.4f updates_per_sec=%.1f\n", (unsigned long long)n, dt.count(),
                n / dt.count());
    if (argc > 3 && std::string(argv[3]) != "-") alg.write_binary(argv[3]);
  } catch (std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
