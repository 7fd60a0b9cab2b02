// gs_gen.cu - seeded synthetic edge streams (benchmark / test inputs, not reference code).
//
// R-MAT(a, b, c, d=1-a-b-c) over 2^log2_v vertices as a counter-based stream: record i is a
// pure function of (seed, i), so any slice [first, first+n) can be generated on the device in
// parallel and the host produces the identical records.  A `delete_frac` share of the records
// (never record 0) re-emits the edge of an earlier insert record j < i, i.e. deletes a
// previously inserted edge under the XOR-toggle semantics of the sketches.  Self-loops are
// resampled (up to 64 draws, then the partner's low bit is flipped).
#include <cmath>

#include "gs_internal.h"

namespace {

GS_HD uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// k-th 64-bit draw of record i
GS_HD uint64_t draw(uint64_t seed, uint64_t i, uint64_t k) {
  return splitmix64(splitmix64(seed ^ (i * 0xD1B54A32D192ED03ULL)) + k * 0x9E3779B97F4A7C15ULL);
}

struct RmatParams {
  uint64_t seed;
  uint32_t log2_v;
  uint32_t tA, tAB, tABC;  // 16-bit quadrant thresholds
  uint32_t tDel;           // 32-bit delete threshold
};

GS_HD void rmat_edge(const RmatParams& p, uint64_t i, uint32_t* ou, uint32_t* ov) {
  uint32_t u = 0, v = 0;
  for (uint32_t a = 0; a < 64; a++) {
    u = 0; v = 0;
    uint64_t r = 0;
    for (uint32_t l = 0; l < p.log2_v; l++) {
      if ((l & 3u) == 0) r = draw(p.seed, i, 16 + (l >> 2) + 8ull * a);
      const uint32_t q = (uint32_t)(r & 0xffffu);
      r >>= 16;
      const uint32_t qu = q >= p.tAB ? 1u : 0u;
      const uint32_t qv = (q >= p.tA && q < p.tAB) || q >= p.tABC ? 1u : 0u;
      u = (u << 1) | qu;
      v = (v << 1) | qv;
    }
    if (u != v) break;
  }
  if (u == v) v ^= 1u;  // log2_v >= 1
  *ou = u;
  *ov = v;
}

GS_HD bool is_delete(const RmatParams& p, uint64_t i) {
  return i > 0 && (uint32_t)draw(p.seed, i, 1) < p.tDel;
}

GS_HD void rmat_record(const RmatParams& p, uint64_t i, uint32_t* u, uint32_t* v) {
  uint64_t j = i;
  if (is_delete(p, i)) {
    j = draw(p.seed, i, 2) % i;
    while (j > 0 && is_delete(p, j)) j--;
  }
  rmat_edge(p, j, u, v);
}

__global__ void k_gen_rmat(RmatParams p, uint64_t first, uint64_t n, uint2* __restrict__ out) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u, v;
    rmat_record(p, first + k, &u, &v);
    out[k] = make_uint2(u, v);
  }
}

RmatParams make_params(uint32_t log2_v, double a, double b, double c, double delete_frac, uint64_t seed) {
  RmatParams p;
  p.seed = seed;
  p.log2_v = log2_v;
  p.tA = (uint32_t)llround(a * 65536.0);
  p.tAB = (uint32_t)llround((a + b) * 65536.0);
  p.tABC = (uint32_t)llround((a + b + c) * 65536.0);
  double del = delete_frac < 0 ? 0 : (delete_frac > 1 ? 1 : delete_frac);
  p.tDel = (uint32_t)std::min(4294967295.0, std::floor(del * 4294967296.0));
  return p;
}

}  // namespace

gs_status gs_gen_rmat_device(uint32_t log2_v, double a, double b, double c, double delete_frac, uint64_t seed,
                             uint64_t first, uint64_t n, uint32_t* d_pairs, cudaStream_t s) {
  if (n == 0) return GS_OK;
  RmatParams p = make_params(log2_v, a, b, c, delete_frac, seed);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint64_t blocks = (n + 255) / 256;
  if (blocks > (uint64_t)sms * 32) blocks = (uint64_t)sms * 32;
  k_gen_rmat<<<(unsigned)blocks, 256, 0, s>>>(p, first, n, reinterpret_cast<uint2*>(d_pairs));
  GS_CUDA_TRY(cudaGetLastError());
  return GS_OK;
}

void gs_gen_rmat_host(uint32_t log2_v, double a, double b, double c, double delete_frac, uint64_t seed,
                      uint64_t first, uint64_t n, uint32_t* pairs) {
  RmatParams p = make_params(log2_v, a, b, c, delete_frac, seed);
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < (long long)n; k++) {
    uint32_t u, v;
    rmat_record(p, first + (uint64_t)k, &u, &v);
    pairs[2 * k] = u;
    pairs[2 * k + 1] = v;
  }
}
