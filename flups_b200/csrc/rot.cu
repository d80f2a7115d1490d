// Pointwise spectral curl and Green's multiply of a ROT solve on the full
// spectrum (Solver.cpp:1485-1516, dothemagic_rot.ipp:102-350):
//   u_hat = G (i K x w_hat),  K_d = symbol of (is_d + koffset_d) * kfact,
// with the spectral or finite-difference symbol of the derivative order.
// Used when the last direction runs through the register DFTs: forward DFT
// of the three components into the spectrum array, this kernel, inverse DFT.
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "pass_desc.h"
#include "rot.h"
#include "spectral.cuh"

namespace flb {

template <typename T>
__global__ void __launch_bounds__(256) rot_mult_kernel(const RotArgs A) {
    using C = typename CT<T>::C;
    const MultSpec& G = A.mult;
    const int64_t n0 = A.n[0], n1 = A.n[1], n2 = A.n[2];
    const int64_t per = n0 * n1 * n2;
    const int64_t total = per * A.nbatch;
    C* data = reinterpret_cast<C*>(A.data);
    const T* green = reinterpret_cast<const T*>(G.green);
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < total; id += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = id / per, r = id - b * per;
        int idx[3];
        idx[0] = (int)(r % n0);
        idx[1] = (int)((r / n0) % n1);
        idx[2] = (int)(r / (n0 * n1));
        int64_t go = 0, off = 0;
        double kk[3];
        for (int d = 0; d < 3; ++d) {
            go += (int64_t)gfold(idx[d], G.gfold[d]) * G.gstr[d];
            off += (int64_t)idx[d] * A.str[d];
            kk[d] = (double)symid(idx[d], G.symstart[d]) + G.koffset[d];
        }
        const double g = (double)green[go] * G.normfact;
        auto kc = [&](int d, int c) {
            return make_double2(fd_symbol(G.odiff, kk[d] * G.kfact[d][c][0], G.hgrid[d]),
                                fd_symbol(G.odiff, kk[d] * G.kfact[d][c][1], G.hgrid[d]));
        };
        C* p0 = data + (3 * b + 0) * A.cstr + off;
        C* p1 = data + (3 * b + 1) * A.cstr + off;
        C* p2 = data + (3 * b + 2) * A.cstr + off;
        const double2 f0 = make_double2(p0->x, p0->y);
        const double2 f1 = make_double2(p1->x, p1->y);
        const double2 f2 = make_double2(p2->x, p2->y);
        const double2 r0 = csub(cmul(f2, kc(1, 2)), cmul(f1, kc(2, 1)));
        const double2 r1 = csub(cmul(f0, kc(2, 0)), cmul(f2, kc(0, 2)));
        const double2 r2 = csub(cmul(f1, kc(0, 1)), cmul(f0, kc(1, 0)));
        *p0 = mkc((T)(r0.x * g), (T)(r0.y * g));
        *p1 = mkc((T)(r1.x * g), (T)(r1.y * g));
        *p2 = mkc((T)(r2.x * g), (T)(r2.y * g));
    }
}

cudaError_t launch_rot_mult(const RotArgs& A, int f64, cudaStream_t s) {
    const int64_t total = (int64_t)A.n[0] * A.n[1] * A.n[2] * A.nbatch;
    int64_t nb = (total + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    if (nb < 1) return cudaSuccess;
    if (f64) rot_mult_kernel<double><<<(unsigned)nb, 256, 0, s>>>(A);
    else rot_mult_kernel<float><<<(unsigned)nb, 256, 0, s>>>(A);
    return cudaGetLastError();
}

}  // namespace flb
