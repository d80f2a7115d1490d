// Half-length DCT-I / DST-I row kernels (row_dct_kernel, FAM 1): the real DFT
// of the row's even / odd extension through one register DFT of half its
// length; FP64, and FP32 with the user's doubles on the input side, the
// output side or neither.
#include "fast_dft_impl.cuh"

namespace flb {

cudaError_t launch_dct1_units(int f64, int in64, int out64, int n, const RowArgs& a, int ncomp, cudaStream_t s) {
    return launch_dct_types<1>(f64, in64, out64, n, a, ncomp, s);
}

}  // namespace flb
