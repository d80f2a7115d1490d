// FP32 fused column kernels: forward DFT, Green's multiply, inverse DFT (instantiations).
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_col_f32_m2(int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    return launch_col_shape<float, 2>(sh, L, a, ncomp, s);
}

}  // namespace flb
