// Index and wave-number helpers of the spectral multiply (shared by the
// general line pass and the pointwise curl kernel).
#pragma once
#include <cuda_runtime.h>

namespace flb {

__device__ __forceinline__ int symid(int i, double symstart) {
    // Topology.hpp:415-430 on one direction
    if (symstart == 0.0 || (double)i <= symstart) return i;
    int a = (int)fabs(2.0 * symstart - (double)i);
    return -(a > 1 ? a : 1);
}

__device__ __forceinline__ int gfold(int i, int Mf) { return (Mf > 0 && 2 * i > Mf) ? Mf - i : i; }

__device__ __forceinline__ double fd_symbol(int odiff, double kk, double h) {
    // dothemagic_rot.ipp: spectral or finite-difference equivalent wave number
    if (odiff == 1) return kk;
    const double a = kk * h;
    if (odiff == 2) return sin(a) / h;
    if (odiff == 4) return (4.0 / 3.0) * sin(a) / h - (1.0 / 6.0) * sin(2.0 * a) / h;
    return 1.5 * sin(a) / h - 0.3 * sin(2.0 * a) / h + (1.0 / 30.0) * sin(3.0 * a) / h;
}

}  // namespace flb
