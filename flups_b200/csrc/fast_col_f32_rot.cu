// FP32 ROT column kernels: forward DFT, curl and Green's multiply, inverse DFT (instantiations).
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_col_f32_m3(int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    return launch_rot_shape<float>(sh, L, a, ncomp, s);
}

}  // namespace flb
