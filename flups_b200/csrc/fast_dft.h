// Arguments and launchers of the register-resident power-of-two DFT passes
// (fast_dft.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace flb {

struct ColArgs {
    const void* in;
    void* out;
    int nx;                 // columns along x (complex elements)
    int nin, nout;          // loaded / stored extent along the line (zero beyond nin)
    int64_t in_lstr, in_ostr, in_cstr;     // element strides: along line, outer, component
    int64_t out_lstr, out_ostr, out_cstr;
    int nouter;
    const void* tw;         // W_L^q, q < L (working precision)
    // fused multiply
    const void* green;
    int64_t g_x, g_line, g_outer;          // folded Green strides
    int f_x, f_line, f_outer;              // fold lengths (0 = none)
    double normfact;
};

struct RowArgs {
    const void* in;
    void* out;
    int nrows;              // rows per component
    int n1;                 // rows are (i1, i2) with i1 < n1
    int nin;                // r2c: real inputs (<= L); c2r: complex inputs (L/2+1)
    int nout;               // r2c: complex outputs kept; c2r: reals kept
    int64_t in_s1, in_s2, in_cstr;   // element strides of rows (i1, i2) and component
    int64_t out_s1, out_s2, out_cstr;
    int in_f64, out_f64;
    const void* tw;         // W_L^q, q < L (L = 2 * Lh)
    const void* twh;        // W_Lh^q, q < Lh
};

bool fast_col_supported(int L);
bool fast_row_supported(int L);
cudaError_t launch_fast_col(int f64, int mode, int L, const ColArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_fast_row(int f64, int c2r, int L, const RowArgs& a, int ncomp, cudaStream_t s);

}  // namespace flb
