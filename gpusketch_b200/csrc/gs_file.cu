// gs_file.cu - edge records straight from a binary stream file (gs_ingest_stream_file).
//
// The reference's readers pull 9-byte records out of the file one buffer at a time and push every
// update through the host gutters (include/graph_sketch_driver.h:141-191).  Here the host only moves
// bytes: each slice of the file is read by several threads with pread straight into a page-locked
// staging slot, copied to the device as raw records on the copy stream, and decoded into (src, dst)
// pairs by a kernel; the read and copy of slice k + 1 overlap the decode and ingest of slice k.
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "gs_internal.h"

namespace {

constexpr uint64_t kRecordBytes = 9;  // {u8 type, u32 src, u32 dst}, packed
constexpr uint64_t kHeaderBytes = 12; // {u32 num_vertices, u64 num_updates}

// raw record i at raw + 9 i -> pair i.  The type byte is not needed: every record toggles its edge.
__global__ void k_decode_records(const uint8_t* __restrict__ raw, uint64_t n, uint2* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint8_t* r = raw + kRecordBytes * i + 1;
    const uint32_t src = (uint32_t)r[0] | ((uint32_t)r[1] << 8) | ((uint32_t)r[2] << 16) | ((uint32_t)r[3] << 24);
    const uint32_t dst = (uint32_t)r[4] | ((uint32_t)r[5] << 8) | ((uint32_t)r[6] << 16) | ((uint32_t)r[7] << 24);
    out[i] = make_uint2(src, dst);
  }
}

// reads exactly `bytes` at `off` with `threads` concurrent preads; false on a short read or error
bool pread_parallel(int fd, uint8_t* dst, uint64_t bytes, uint64_t off, int threads) {
  const uint64_t piece = std::max<uint64_t>(1 << 20, (bytes + threads - 1) / threads);
  const int pieces = (int)((bytes + piece - 1) / piece);
  int bad = 0;
#pragma omp parallel for num_threads(threads) reduction(| : bad) schedule(static, 1)
  for (int p = 0; p < pieces; p++) {
    uint64_t done = (uint64_t)p * piece;
    const uint64_t end = std::min(bytes, done + piece);
    while (done < end) {
      const ssize_t r = pread(fd, dst + done, end - done, (off_t)(off + done));
      if (r <= 0) { bad = 1; break; }
      done += (uint64_t)r;
    }
  }
  return bad == 0;
}

struct Fd {
  int fd = -1;
  ~Fd() { if (fd >= 0) close(fd); }
};

}  // namespace

extern "C" gs_status gs_ingest_stream_file(gs_graph* g, const char* path, uint64_t first, uint64_t count,
                                           uint64_t* ingested) {
  if (!g || !path) { gs_set_error("gs_ingest_stream_file: null argument"); return GS_ERR_BAD_ARG; }
  if (ingested) *ingested = 0;
  Fd f;
  f.fd = open(path, O_RDONLY);
  if (f.fd < 0) { gs_set_error(std::string("cannot open stream file ") + path); return GS_ERR_IO; }
  uint8_t hdr[kHeaderBytes];
  if (!pread_parallel(f.fd, hdr, kHeaderBytes, 0, 1)) { gs_set_error("truncated stream header"); return GS_ERR_IO; }
  uint32_t file_v = 0;
  uint64_t file_n = 0;
  std::memcpy(&file_v, hdr, 4);
  std::memcpy(&file_n, hdr + 4, 8);
  if (file_v > g->V) {
    gs_set_error("stream file has " + std::to_string(file_v) + " vertices, the graph " + std::to_string(g->V));
    return GS_ERR_BAD_ARG;
  }
  if (first >= file_n) return GS_OK;
  const uint64_t last = count > file_n - first ? file_n : first + count;
  GsDeviceGuard guard(g->device);
  if (!guard.ok) { gs_set_error("cannot select CUDA device"); return GS_ERR_NO_DEVICE; }
  cudaStream_t s = g->stream;
  g->labels_valid = false;
  g->changes++;
  GS_TRY(gs_ensure_pair_staging(g, ((last - first) * kRecordBytes + 7) / 8));
  const uint64_t slot_bytes = g->pairs_cap * 2 * sizeof(uint32_t);
  const uint64_t per = slot_bytes / kRecordBytes;  // records per slice
  if (!g->d_file_pairs) GS_CUDA_TRY(cudaMalloc(&g->d_file_pairs, per * sizeof(uint2)));
  const int threads = std::max(1, std::min(16, (int)sysconf(_SC_NPROCESSORS_ONLN)));
  uint8_t* hp = static_cast<uint8_t*>(g->h_pin);
  uint8_t* dp = reinterpret_cast<uint8_t*>(g->d_pairs);
  for (uint64_t at = first, k = 0; at < last; k++) {
    const uint64_t m = std::min(per, last - at);
    const int slot = (int)(k & 1);
    // the page-locked slot is free once its previous copy has landed
    GS_CUDA_TRY(cudaEventSynchronize(g->ev_copy[slot]));
    if (!pread_parallel(f.fd, hp + slot * slot_bytes, m * kRecordBytes, kHeaderBytes + at * kRecordBytes, threads)) {
      GS_CUDA_TRY(cudaStreamSynchronize(s));
      gs_set_error(std::string("stream file read failed or truncated: ") + path);
      return GS_ERR_IO;
    }
    // the device slot is free once the decode of its previous slice has read it
    GS_CUDA_TRY(cudaStreamWaitEvent(g->copy_stream, g->ev_done[slot], 0));
    GS_CUDA_TRY(cudaMemcpyAsync(dp + slot * slot_bytes, hp + slot * slot_bytes, m * kRecordBytes,
                                cudaMemcpyHostToDevice, g->copy_stream));
    GS_CUDA_TRY(cudaEventRecord(g->ev_copy[slot], g->copy_stream));
    GS_CUDA_TRY(cudaStreamWaitEvent(s, g->ev_copy[slot], 0));
    const int grid = (int)std::min<uint64_t>((m + 255) / 256, (uint64_t)g->num_sms * 8);
    k_decode_records<<<grid, 256, 0, s>>>(dp + slot * slot_bytes, m, g->d_file_pairs);
    GS_CUDA_TRY(cudaGetLastError());
    GS_CUDA_TRY(cudaEventRecord(g->ev_done[slot], s));
    GS_TRY(gs_ingest_device_pairs(g, reinterpret_cast<const uint32_t*>(g->d_file_pairs), m, -1, s));
    at += m;
    if (ingested) *ingested += m;
  }
  GS_CUDA_TRY(cudaStreamSynchronize(g->copy_stream));
  return GS_OK;
}
