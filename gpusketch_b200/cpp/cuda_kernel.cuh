// cuda_kernel.cuh - the part of the reference's include/cuda_kernel.cuh that its tools use next to the
// algorithm classes: the SketchParams they fill (declared in gpusketch_types.h), the CUDA error-check
// macro and the device integer typedefs.  The reference's sketch-update kernel itself has no
// counterpart here: the library's kernels sit behind the C ABI of include/gpusketch.h.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#include "gpusketch_types.h"

typedef unsigned long long int uint64_cu;
typedef uint64_cu vec_t_cu;

// include/cuda_kernel.cuh:11-21: report a failed CUDA runtime call of the caller and exit
#define gpuErrchk(ans) { gpuAssert((ans), __FILE__, __LINE__); }
inline void gpuAssert(cudaError_t code, const char* file, int line, bool abort = true) {
  if (code != cudaSuccess) {
    std::fprintf(stderr, "GPUassert: %s %s %d\n", cudaGetErrorString(code), file, line);
    if (abort) std::exit(code);
  }
}
