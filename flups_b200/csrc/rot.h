// Pointwise curl-and-Green kernel of the ROT solve on the full spectrum (rot.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pass_desc.h"

namespace flb {

struct RotArgs {
    void* data;          // spectrum, working-precision complex, 3 components per batch
    int n[3];            // extents (x fastest)
    int64_t str[3];      // element strides
    int64_t cstr;        // component stride
    int nbatch;
    MultSpec mult;       // mode 2 fields: Green, folds, wave-number tables, derivative order
};

cudaError_t launch_rot_mult(const RotArgs& A, int f64, cudaStream_t s);

}  // namespace flb
