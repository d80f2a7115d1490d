// r2r row kernels (DCT / DST I-IV), instantiations: FP64, and FP32 with the
// user's doubles on the input side (first pass) or the output side (last pass).
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_r2r_units(int f64, int in64, int out64, int M, const RowArgs& a, int ncomp, cudaStream_t s) {
    if (f64) return launch_r2r_len<double, double, double>(M, a, ncomp, s);
    if (in64 && !out64) return launch_r2r_len<float, double, float>(M, a, ncomp, s);
    if (!in64 && out64) return launch_r2r_len<float, float, double>(M, a, ncomp, s);
    if (!in64 && !out64) return launch_r2r_len<float, float, float>(M, a, ncomp, s);
    return cudaErrorInvalidValue;
}

}  // namespace flb
