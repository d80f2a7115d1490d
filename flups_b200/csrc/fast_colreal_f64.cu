// F64 column r2c / c2r kernels (instantiations).
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_colreal_f64(int c2r, int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    if (c2r) return launch_colreal_shape<double, double, true>(sh, L, a, ncomp, s);
    return launch_colreal_shape<double, double, false>(sh, L, a, ncomp, s);
}

}  // namespace flb
