// FP64 column DFT kernels, forward and inverse (instantiations).
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_col_f64_m01(int mode, int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    if (mode == 0) return launch_col_shape<double, 0>(sh, L, a, ncomp, s);
    return launch_col_shape<double, 1>(sh, L, a, ncomp, s);
}

}  // namespace flb
