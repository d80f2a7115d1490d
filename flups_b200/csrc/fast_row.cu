// Row (x) r2c / c2r kernels (instantiations).  xt64: the real side is the
// user's doubles (FP32 mode) rather than the working precision.
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_row_units(int f64, int c2r, int xt64, bool half, int L, const RowArgs& a, int ncomp, cudaStream_t s) {
    if (f64) {
        if (c2r) return launch_row_half<double, double, true>(half, L, a, ncomp, s);
        return launch_row_half<double, double, false>(half, L, a, ncomp, s);
    }
    if (c2r) {
        if (xt64) return launch_row_half<float, double, true>(half, L, a, ncomp, s);
        return launch_row_half<float, float, true>(half, L, a, ncomp, s);
    }
    if (xt64) return launch_row_half<float, double, false>(half, L, a, ncomp, s);
    return launch_row_half<float, float, false>(half, L, a, ncomp, s);
}

}  // namespace flb
