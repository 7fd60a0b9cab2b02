// gs_common.cuh - types, hashing and error plumbing shared by the sm_100a kernels and the host.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <cuda_runtime.h>

#include "../../include/gpusketch.h"

#if defined(__CUDACC__)
#define GS_HD __host__ __device__ __forceinline__
#else
#define GS_HD inline
#endif

// Bucket {alpha, gamma} (include/bucket.h:7-12).  16-byte aligned so a bucket moves as one
// 128-bit load/store; the reference packs the same two u64s, so the byte layout is identical.
struct alignas(16) GsBucket {
  uint64_t alpha;
  uint64_t gamma;
};
static_assert(sizeof(GsBucket) == 16, "bucket must be 16 bytes");

// ----------------------------------------------------------------------------------------
// XXH3_64bits_withSeed on an 8-byte little-endian key (include/types.h:8-9), restated from the
// published xxHash algorithm (XXH3_len_4to8_64b followed by the rrmxmx avalanche).
//
// With k' = (key >> 32) | (key << 32) and B(seed) = kSecret64[8..16) ^ kSecret64[16..24) - seed',
// the first mixing step x = y ^ rotl(y,49) ^ rotl(y,24) of y = k' ^ B is linear over XOR, so
//     x = mix(k') ^ mix(B(seed)),   mix(z) = z ^ rotl(z,49) ^ rotl(z,24).
// mix(k') depends only on the edge, mix(B) only on the seed: the ingest kernel computes mix(k')
// once per record and each column's hash is one XOR plus the two multiplies of gs_hash_tail.
// ----------------------------------------------------------------------------------------
constexpr uint64_t kGsSecret8to24 = 0x1cad21f72c81017cULL ^ 0xdb979083e96dd4deULL;
constexpr uint64_t kGsMx2 = 0x9FB21C651E98DF25ULL;

GS_HD uint64_t gs_rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

GS_HD uint64_t gs_mix(uint64_t z) { return z ^ gs_rotl64(z, 49) ^ gs_rotl64(z, 24); }

// mix(k') for key k
GS_HD uint64_t gs_key_mix(uint64_t key) { return gs_mix((key >> 32) | (key << 32)); }

// Inverse of gs_mix.  mix is the GF(2)-linear map M = I + R^49 + R^24 (R = rotate left by one);
// squaring commuting terms gives M^(2^k) = I + R^(49*2^k) + R^(24*2^k), so M^8 = R^8, M^16 = R^16,
// M^32 = R^32, M^64 = I and M^-1 = M^63 = M * M^2 * M^4 * R^56.
GS_HD uint64_t gs_mix_inv(uint64_t z) {
  z = z ^ gs_rotl64(z, 49) ^ gs_rotl64(z, 24);
  z = z ^ gs_rotl64(z, 34) ^ gs_rotl64(z, 48);
  z = z ^ gs_rotl64(z, 4) ^ gs_rotl64(z, 32);
  return gs_rotl64(z, 56);
}

// key k from gs_key_mix(k); both maps are XOR-linear, so a XOR of mixed keys unmixes to the XOR
// of the keys
GS_HD uint64_t gs_key_unmix(uint64_t mixed) {
  const uint64_t k = gs_mix_inv(mixed);
  return (k >> 32) | (k << 32);
}

// mix(B(seed)) for seed s
GS_HD uint64_t gs_seed_mix(uint64_t seed) {
  uint32_t lo = (uint32_t)seed;
  uint32_t sw = ((lo & 0xffu) << 24) | ((lo & 0xff00u) << 8) | ((lo >> 8) & 0xff00u) | (lo >> 24);
  uint64_t s = seed ^ ((uint64_t)sw << 32);
  return gs_mix(kGsSecret8to24 - s);
}

// rrmxmx after the rotate-xor step: h = x*M; h ^= (h>>35)+8; h *= M; return h ^ (h>>28).
// (h>>35) < 2^29, so +8 never carries out of the low word and the xor only touches it.
GS_HD uint64_t gs_hash_tail(uint64_t x) {
  uint64_t h = x * kGsMx2;
  uint32_t lo = (uint32_t)h, hi = (uint32_t)(h >> 32);
  lo ^= (hi >> 3) + 8u;
  h = ((uint64_t)hi << 32) | lo;
  h *= kGsMx2;
  return h ^ (h >> 28);
}

GS_HD uint64_t gs_xxh3_8(uint64_t key, uint64_t seed) {
  return gs_hash_tail(gs_key_mix(key) ^ gs_seed_mix(seed));
}

// concat_pairing_fn (src/util.cpp:45-51)
GS_HD uint64_t gs_concat(uint32_t a, uint32_t b) {
  uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
  return ((uint64_t)lo << 32) | hi;
}

#if defined(__CUDACC__)
// ctz(hash | 1<<max_depth) = min(ctz(hash), max_depth), from the tail of the hash
// (Bucket_Boruvka::get_index_depth, include/bucket.h:54-59).  Computes only the low word of the
// final xorshift unless it is zero (probability 2^-32).
__device__ __forceinline__ uint32_t gs_depth_from_mixed(uint64_t x, uint32_t max_depth) {
  // (hi >> 3) + 8 is written as umulhi(hi, 2^29) + 8, one multiply-add on the FMA pipe next to the
  // 64-bit products; the low word of (h2:l2) >> 28 is one funnel shift
  uint64_t h = x * kGsMx2;
  uint32_t lo = (uint32_t)h, hi = (uint32_t)(h >> 32);
  lo ^= __umulhi(hi, 1u << 29) + 8u;
  h = ((uint64_t)hi << 32) | lo;
  h *= kGsMx2;
  const uint32_t l2 = (uint32_t)h, h2 = (uint32_t)(h >> 32);
  const uint32_t flo = l2 ^ __funnelshift_r(l2, h2, 28);
  // ctz of the 64-bit value: the high word only decides when the low word is zero (probability
  // 2^-32), so it is computed in a branch that practically never runs
  uint32_t d = (uint32_t)__ffs((int)flo) - 1u;
  if (__builtin_expect(flo == 0u, 0)) d = 32u + __clz(__brev(h2 ^ (h2 >> 28)));  // 64 for a zero hash
  return d < max_depth ? d : max_depth;
}

// The same depth in two steps, for loops that cap the depth anyway.  gs_depth_low returns the ctz of
// the final hash's low word, exact whenever that word is non-zero, and ~0u when it is zero
// (probability 2^-32), with the high product word in *h2; gs_depth_finish completes a low-word depth
// of 32 or more from the high word and caps it at max_depth.  (__ffs is one instruction fewer than
// __clz(__brev()), and its ffs(0) - 1 = ~0u is exactly the "look at the high word" signal.)
__device__ __forceinline__ uint32_t gs_depth_low(uint64_t x, uint32_t* h2_out) {
  uint64_t h = x * kGsMx2;
  uint32_t lo = (uint32_t)h, hi = (uint32_t)(h >> 32);
  lo ^= __umulhi(hi, 1u << 29) + 8u;
  h = ((uint64_t)hi << 32) | lo;
  h *= kGsMx2;
  const uint32_t l2 = (uint32_t)h, h2 = (uint32_t)(h >> 32);
  *h2_out = h2;
  return (uint32_t)__ffs((int)(l2 ^ __funnelshift_r(l2, h2, 28))) - 1u;
}

// min(ctz(final hash's low word), cap) for capbit = 1 << cap, cap < 32: the cap bit is OR-ed in by the
// same three-input logic op as the xorshift, so the capped depth costs no instruction more than the
// uncapped one.  A result of cap means "cap or deeper".
__device__ __forceinline__ uint32_t gs_depth_capped(uint64_t x, uint32_t capbit) {
  uint64_t h = x * kGsMx2;
  uint32_t lo = (uint32_t)h, hi = (uint32_t)(h >> 32);
  lo ^= __umulhi(hi, 1u << 29) + 8u;
  h = ((uint64_t)hi << 32) | lo;
  h *= kGsMx2;
  const uint32_t l2 = (uint32_t)h, h2 = (uint32_t)(h >> 32);
  return (uint32_t)__ffs((int)((l2 ^ __funnelshift_r(l2, h2, 28)) | capbit)) - 1u;
}

__device__ __forceinline__ uint32_t gs_depth_finish(uint32_t d_low, uint32_t h2, uint32_t max_depth) {
  const uint32_t d = d_low < 32u ? d_low : 32u + __clz(__brev(h2 ^ (h2 >> 28)));  // 64 for a zero hash
  return d < max_depth ? d : max_depth;
}
#endif

// ----------------------------------------------------------------------------------------
// Sketch geometry (include/sketch.h:177-191,312-320; src/sketch.cpp:24-30)
// ----------------------------------------------------------------------------------------
struct GsGeom {
  uint32_t V;
  uint32_t num_samples;
  uint32_t num_columns;
  uint32_t bkt_per_col;
  uint32_t num_buckets;
};

GsGeom gs_make_geom(uint32_t V, double sketches_factor);

// Thread-local error message behind gs_last_error().
void gs_set_error(const std::string& msg);

// the file name of a source path, for error messages
inline const char* gs_source_name(const char* path) {
  const char* base = path;
  for (const char* p = path; *p; ++p)
    if (*p == '/') base = p + 1;
  return base;
}

#define GS_CUDA_TRY(expr)                                                                    \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess) {                                                                 \
      gs_set_error(std::string(#expr) + ": " + cudaGetErrorString(_e) + " @" +                \
                   gs_source_name(__FILE__) + ":" + std::to_string(__LINE__));               \
      return _e == cudaErrorMemoryAllocation ? GS_ERR_OOM : GS_ERR_CUDA;                     \
    }                                                                                        \
  } while (0)

#define GS_TRY(expr)                     \
  do {                                   \
    gs_status _s = (expr);               \
    if (_s != GS_OK) return _s;          \
  } while (0)

// Device-side error word bits (read back by the host after a phase).
enum : uint32_t {
  GS_DEV_ERR_VERTEX_RANGE = 1u,   // an input vertex id >= V
  GS_DEV_ERR_CAPACITY = 2u,       // more records than the scratch holds
  GS_DEV_ERR_DSU_LIMIT = 4u,      // a DSU walk exceeded its iteration bound
  GS_DEV_ERR_TIMEOUT = 8u,        // a bounded device-side wait (grid barrier) gave up
};
