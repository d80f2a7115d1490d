// Pointwise Green (STD) and curl-and-Green (ROT) multiplies on the full spectrum (rot.cu).
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
    int nbatch;          // ROT: groups of 3 components
    int ncomp;           // STD: components multiplied
    MultSpec mult;       // mode 1 (STD) or 2 (ROT): Green, folds, wave-number tables, derivative order
};

// data in FP64 or the working precision, Green in the working precision
cudaError_t launch_spec_mult(const RotArgs& A, int data_f64, int green_f64, cudaStream_t s);
// the curl's wave-number symbols K_{d,c}(i), i < n[d], of a ROT multiply
// (mode 2 MultSpec), table (d, c) at out + (3 d + c) kstr complex values of
// the working precision
cudaError_t launch_ksym_table(const MultSpec& G, const int n[3], int kstr, void* out, int f64, cudaStream_t s);

}  // namespace flb
