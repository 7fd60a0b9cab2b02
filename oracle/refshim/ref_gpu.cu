// Test oracle, not part of the product: extern "C" entry points over the reference's own GPU
// sketch-update kernel (CudaKernel::sketchUpdate, src/cuda_kernel.cu:152-257 of the reference),
// which oracle/Makefile compiles for sm_100a where the source lies.  The GPU tests use it to check
// that the library's device sketches equal the XOR of the reference kernel's per-batch deltas, and to
// time that kernel on the same records.  Nothing in the library links it.
#include <cstdint>

#include "cuda_kernel.cuh"

// CudaKernel::updateSharedMemory: the reference raises the kernels' dynamic shared-memory limit to one
// delta sketch (num_buckets * (8 + 8) bytes) before its first launch (include/cuda_stream.h:78-80).
extern "C" int gsref_gpu_prepare(uint64_t num_buckets) {
  CudaKernel k;
  k.updateSharedMemory((size_t)num_buckets * (sizeof(vec_t_cu) + sizeof(vec_hash_t)));
  return (int)cudaGetLastError();
}

// One launch of the reference kernel: block b builds the delta sketch of batch b (vertex src[b],
// neighbours dsts[start[b] .. start[b] + sizes[b])) in shared memory and writes it to
// deltas[b * num_buckets ..], as CudaStream::process_batch_default does (include/cuda_stream.h:137).
extern "C" int gsref_gpu_sketch_update(int num_threads, int num_batches, void* stream, uint32_t* d_dsts,
                                       uint32_t* d_src, uint64_t* d_sizes, uint64_t* d_start, uint64_t num_samples,
                                       uint64_t num_buckets, uint64_t num_columns, uint64_t bkt_per_col,
                                       uint64_t seed, void* d_deltas) {
  CudaKernel k;
  SketchParams p{};
  p.num_samples = num_samples;
  p.num_buckets = num_buckets;
  p.num_columns = num_columns;
  p.bkt_per_col = bkt_per_col;
  p.seed = seed;
  p.cudaUVM_enabled = false;
  p.cudaUVM_buckets = nullptr;
  p.d_buckets = static_cast<Bucket*>(d_deltas);
  k.sketchUpdate(num_threads, num_batches, static_cast<cudaStream_t>(stream), d_dsts, d_src,
                 reinterpret_cast<vec_t*>(d_sizes), reinterpret_cast<vec_t*>(d_start), p);
  return (int)cudaGetLastError();
}
