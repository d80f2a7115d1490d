// Pointwise spectral multiplies on the full spectrum (Solver.cpp:1471-1516):
//   STD (mode 1): f_hat <- G f_hat                       (dothemagic_std.ipp:56-83)
//   ROT (mode 2): u_hat <- G (i K x w_hat), K_d = symbol of (is_d + koffset_d) kfact
//                 with the spectral or finite-difference symbol of the derivative
//                 order (dothemagic_rot.ipp:102-350)
// G is the stored folded spectrum (normfact and volfact included).  Used by the
// split ROT solve (forward DFT into the spectrum, this kernel, inverse DFT) and
// by flups_do_mult, whose data are the user's doubles while G is in the working
// precision.
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "pass_desc.h"
#include "rot.h"
#include "spectral.cuh"

namespace flb {

template <typename TD, typename TG>
__global__ void __launch_bounds__(256) spec_mult_kernel(const RotArgs A) {
    using C = typename CT<TD>::C;
    const MultSpec& G = A.mult;
    const int64_t n0 = A.n[0], n1 = A.n[1], n2 = A.n[2];
    const int64_t per = n0 * n1 * n2;
    const int64_t groups = (G.mode == 2) ? A.nbatch : A.ncomp;  // ROT: 3 components per group
    const int64_t total = per * groups;
    C* data = reinterpret_cast<C*>(A.data);
    const TG* green = reinterpret_cast<const TG*>(G.green);
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < total; id += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = id / per, r = id - b * per;
        int idx[3];
        idx[0] = (int)(r % n0);
        idx[1] = (int)((r / n0) % n1);
        idx[2] = (int)(r / (n0 * n1));
        int64_t go = 0, off = 0;
        for (int d = 0; d < 3; ++d) {
            go += (int64_t)gfold(idx[d], G.gfold[d]) * G.gstr[d];
            off += (int64_t)idx[d] * A.str[d];
        }
        const double g = (double)green[go] * G.normfact;
        if (G.mode != 2) {
            C* p = data + b * A.cstr + off;
            *p = mkc((TD)(p->x * g), (TD)(p->y * g));
            continue;
        }
        double kk[3];
        for (int d = 0; d < 3; ++d) kk[d] = (double)symid(idx[d], G.symstart[d]) + G.koffset[d];
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
        *p0 = mkc((TD)(r0.x * g), (TD)(r0.y * g));
        *p1 = mkc((TD)(r1.x * g), (TD)(r1.y * g));
        *p2 = mkc((TD)(r2.x * g), (TD)(r2.y * g));
    }
}

cudaError_t launch_spec_mult(const RotArgs& A, int data_f64, int green_f64, cudaStream_t s) {
    const int64_t groups = (A.mult.mode == 2) ? A.nbatch : A.ncomp;
    const int64_t total = (int64_t)A.n[0] * A.n[1] * A.n[2] * groups;
    int64_t nb = (total + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    if (nb < 1) return cudaSuccess;
    if (data_f64 && green_f64) spec_mult_kernel<double, double><<<(unsigned)nb, 256, 0, s>>>(A);
    else if (data_f64) spec_mult_kernel<double, float><<<(unsigned)nb, 256, 0, s>>>(A);
    else spec_mult_kernel<float, float><<<(unsigned)nb, 256, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_rot_mult(const RotArgs& A, int f64, cudaStream_t s) { return launch_spec_mult(A, f64, f64, s); }

}  // namespace flb
