// gs_noalloc.cu - edge-record ingest that allocates nothing.
//
// Some callers cannot allocate device memory: their device memory is owned by another allocator
// (a framework's caching allocator, an embedded runtime that forbids allocation once it has
// started), so every cudaMalloc would step outside the budget they were given.  This entry point
// serves them: the caller passes the records and its own sketch buffer, and every scratch buffer of
// the bucketing passes and the sketch update lives in one file-scope device array, sized for at
// most GS_NOALLOC_MAX_VERTICES vertices and GS_NOALLOC_MAX_EDGES records per call.  Every GPU that
// loads the library holds that array (about 2.3 MB) until the process exits.
//
// In host code the name g_noalloc_scratch is only a host-side stand-in for the array: every call
// asks the runtime for the array's device address on the current device (cudaGetSymbolAddress, with
// that device current) and hands that address to the kernels.  Resolving it per call costs a few
// microseconds and stays right after cudaDeviceReset, which reloads the module at a new address.
// All calls share the one array and it keeps the last call's contents, so calls on the same device
// that overlap on the GPU (different streams, or different host threads) race on it.  A call waits
// for its own stream before it returns (it reads the device error word back), so it cannot be made
// while that stream is being captured into a CUDA graph.
#include "gs_internal.h"

namespace {

constexpr uint64_t kMaxV = GS_NOALLOC_MAX_VERTICES;
constexpr uint64_t kMaxRecords = 2ull * GS_NOALLOC_MAX_EDGES;
constexpr uint32_t kPartLb = 9;  // the bucketing split for V <= 2^16: 2^16 / 2^9 = 128 buckets
constexpr uint64_t kMaxBuckets = (kMaxV + (1u << kPartLb) - 1) >> kPartLb;
constexpr uint64_t kScanTileElems = 4096;

constexpr uint64_t al256(uint64_t x) { return (x + 255) & ~255ull; }

// byte offsets of the scratch buffers
constexpr uint64_t kOffStatus = 0;
constexpr uint64_t kOffColmix = kOffStatus + al256(16 * 4);
constexpr uint64_t kOffCnt = kOffColmix + al256(65 * 8);
constexpr uint64_t kOffOff = kOffCnt + al256((kMaxV + 1) * 4);
constexpr uint64_t kOffChoff = kOffOff + al256((kMaxV + 1) * 4);
constexpr uint64_t kOffTile = kOffChoff + al256((kMaxV + 1) * 4);
constexpr uint64_t kOffBkt = kOffTile + al256(2 * ((kMaxV + kScanTileElems - 1) / kScanTileElems + 1) * 4);
constexpr uint64_t kOffPart = kOffBkt + al256((4 * kMaxBuckets + 2) * 4);
constexpr uint64_t kOffNbr = kOffPart + al256(kMaxRecords * 8);
constexpr uint64_t kScratchBytes = kOffNbr + al256(kMaxRecords * 4);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// device address of the scratch array on the current device, and the device's SM count
gs_status scratch_for_current_device(unsigned char** out, int* sms) {
  int dev = 0;
  GS_CUDA_TRY(cudaGetDevice(&dev));
  void* p = nullptr;
  GS_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  int n = 0;
  GS_CUDA_TRY(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  *out = static_cast<unsigned char*>(p);
  *sms = n > 0 ? n : 1;
  return GS_OK;
}

// per-column hash constants mix(B(seed+5c)) and the checksum constant mix(B(seed)) at [C]
__global__ void k_noalloc_colmix(uint64_t* colmix, uint32_t C, uint64_t seed) {
  for (uint32_t c = threadIdx.x; c <= C; c += blockDim.x)
    colmix[c] = gs_seed_mix(c < C ? seed + 5ull * c : seed);
}

}  // namespace

extern "C" gs_status gs_ingest_pairs_noalloc(uint32_t num_vertices, uint64_t seed, double sketches_factor,
                                             const uint32_t* pairs, uint64_t n, gs_bucket* sketches,
                                             void* cuda_stream) {
  if (num_vertices < 2 || num_vertices > GS_NOALLOC_MAX_VERTICES) {
    gs_set_error("gs_ingest_pairs_noalloc: num_vertices must be in [2, " + std::to_string(GS_NOALLOC_MAX_VERTICES) +
                 "], got " + std::to_string(num_vertices));
    return GS_ERR_BAD_ARG;
  }
  if (n > GS_NOALLOC_MAX_EDGES) {
    gs_set_error("gs_ingest_pairs_noalloc: at most " + std::to_string(GS_NOALLOC_MAX_EDGES) +
                 " edge records per call, got " + std::to_string(n));
    return GS_ERR_BAD_ARG;
  }
  if (!sketches || (n && !pairs)) {
    gs_set_error("gs_ingest_pairs_noalloc: null pointer");
    return GS_ERR_BAD_ARG;
  }
  const GsGeom geom = gs_make_geom(num_vertices, sketches_factor > 0 ? sketches_factor : 1.0);
  if (geom.num_columns > 64) {
    gs_set_error("gs_ingest_pairs_noalloc: more than 64 sketch columns are not supported");
    return GS_ERR_BAD_ARG;
  }
  if (n == 0) return GS_OK;

  unsigned char* base = nullptr;
  int sms = 0;
  GS_TRY(scratch_for_current_device(&base, &sms));
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);

  GsScratchIngest x;
  x.pairs = pairs;
  x.n = n;
  x.sketches = reinterpret_cast<GsBucket*>(sketches);
  x.geom = geom;
  x.colmix = reinterpret_cast<const uint64_t*>(base + kOffColmix);
  x.status = reinterpret_cast<uint32_t*>(base + kOffStatus);
  x.cnt = reinterpret_cast<uint32_t*>(base + kOffCnt);
  x.off = reinterpret_cast<uint32_t*>(base + kOffOff);
  x.choff = reinterpret_cast<uint32_t*>(base + kOffChoff);
  x.tile = reinterpret_cast<uint32_t*>(base + kOffTile);
  x.bkt = reinterpret_cast<uint32_t*>(base + kOffBkt);
  x.part = reinterpret_cast<uint2*>(base + kOffPart);
  x.nbr = reinterpret_cast<uint32_t*>(base + kOffNbr);
  x.records_cap = kMaxRecords;
  x.part_lb = kPartLb;
  x.part_buckets = (num_vertices + (1u << kPartLb) - 1) >> kPartLb;
  x.num_sms = sms;
  x.chunk = 1024;
  x.warps = 4;

  k_noalloc_colmix<<<1, 128, 0, s>>>(reinterpret_cast<uint64_t*>(base + kOffColmix), geom.num_columns, seed);
  GS_CUDA_TRY(cudaGetLastError());
  GS_TRY(gs_ingest_pairs_on_scratch(x, s));
  // the call returns once the update is applied, with the device error word checked
  uint32_t err = 0;
  GS_CUDA_TRY(cudaMemcpyAsync(&err, x.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  GS_CUDA_TRY(cudaStreamSynchronize(s));
  if (err & GS_DEV_ERR_VERTEX_RANGE) {
    gs_set_error("gs_ingest_pairs_noalloc: a record named a vertex id >= num_vertices; it was skipped and every "
                 "other record of the call was applied");
    return GS_ERR_BAD_ARG;
  }
  if (err) {
    gs_set_error("gs_ingest_pairs_noalloc: device consistency check failed");
    return GS_ERR_INTERNAL;
  }
  return GS_OK;
}
