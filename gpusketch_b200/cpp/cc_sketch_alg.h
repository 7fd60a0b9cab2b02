// cc_sketch_alg.h - the reference's include/cc_sketch_alg.h name: CCSketchAlg, the CPU connected-
// components algorithm of the reference, is the same device implementation here (an alias of
// CCGPUSketchAlg, cc_gpu_sketch_alg.h), so tools that include this header build unchanged.
#pragma once

#include "cc_gpu_sketch_alg.h"
