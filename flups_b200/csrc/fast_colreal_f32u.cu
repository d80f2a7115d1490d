// FP32 column r2c / c2r kernels whose real side is the user's doubles: the
// first (r2c) and last (c2r) passes of a solve that starts with a column
// direction (instantiations).
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_colreal_f32u(int c2r, int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    if (c2r) return launch_colreal_shape<float, double, true>(sh, L, a, ncomp, s);
    return launch_colreal_shape<float, double, false>(sh, L, a, ncomp, s);
}

}  // namespace flb
