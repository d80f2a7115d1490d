// F64 fused row kernels of the last direction along x (instantiations).
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_rowfused_f64(int rot, int sh, int L, const RowFusedArgs& a, int ncomp, cudaStream_t s) {
    if (rot) return launch_row_fused_shape<double, true>(sh, L, a, ncomp, s);
    return launch_row_fused_shape<double, false>(sh, L, a, ncomp, s);
}

}  // namespace flb
