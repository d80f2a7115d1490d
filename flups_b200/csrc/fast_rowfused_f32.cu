// F32 fused row kernels of the last direction along x (instantiations).
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_rowfused_f32(int rot, int sh, int L, const RowFusedArgs& a, int ncomp, cudaStream_t s) {
    if (rot) return launch_row_fused_shape<float, true>(sh, L, a, ncomp, s);
    return launch_row_fused_shape<float, false>(sh, L, a, ncomp, s);
}

}  // namespace flb
