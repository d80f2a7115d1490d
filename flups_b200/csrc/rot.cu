// Pointwise spectral multiplies on the full spectrum (Solver.cpp:1471-1516):
//   STD (mode 1): f_hat <- G f_hat                       (dothemagic_std.ipp:56-83)
//   ROT (mode 2): u_hat <- G (i K x w_hat), K_d = symbol of (is_d + koffset_d) kfact
//                 with the spectral or finite-difference symbol of the derivative
//                 order (dothemagic_rot.ipp:102-350)
// G is the stored folded spectrum (normfact and volfact included).  Used by
// flups_do_mult, whose data are the user's doubles while G is in the working
// precision (a solve multiplies inside its last-direction pass instead).
// ksym_kernel builds the curl symbols that the fused ROT column pass reads.
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "pass_desc.h"
#include "rot.h"
#include "spectral.cuh"

namespace flb {

// Block = 128 x-positions of one y row and a chunk of zb z values (of one
// component for STD, of one 3-component group for ROT): no index division per element, the
// x and y parts of the wave numbers and of the Green's index are computed
// once per thread, the z part once per z.  Wave numbers
// are evaluated in FP64 and rounded once to the data precision, in which the
// per-element curl and scaling run.
template <typename TD, typename TG>
__global__ void __launch_bounds__(128) spec_mult_kernel(const __grid_constant__ RotArgs A, int zb) {
    using C = typename CT<TD>::C;
    using T = TD;
    const MultSpec& G = A.mult;
    // thread = x, loop over z one by one
    const int x = blockIdx.x * 128 + threadIdx.x;
    if (x >= A.n[0]) return;
    const int y = blockIdx.y;
    const int nzc = (A.n[2] + zb - 1) / zb;
    const int grp = blockIdx.z / nzc, z0 = (blockIdx.z % nzc) * zb;
    const int z1 = min((blockIdx.z % nzc) * zb + zb, A.n[2]);
    const TG* green = reinterpret_cast<const TG*>(G.green);
    const int64_t gxy = (int64_t)gfold(x, G.gfold[0]) * G.gstr[0] + (int64_t)gfold(y, G.gfold[1]) * G.gstr[1];
    const int64_t ox = (int64_t)x * A.str[0];
    const int64_t oxy = ox + (int64_t)y * A.str[1];
    C* data = reinterpret_cast<C*>(A.data);
    if (G.mode != 2) {
        C* p = data + grp * A.cstr + oxy;
        for (int z = z0; z < z1; ++z) {
            const double g = (double)green[gxy + (int64_t)gfold(z, G.gfold[2]) * G.gstr[2]] * G.normfact;
            C* q = p + (int64_t)z * A.str[2];
            *q = mkc((TD)(q->x * g), (TD)(q->y * g));
        }
        return;
    }
    // K_d for component c: (symbol((is_d + koffset_d) kfact_dc0), symbol(... kfact_dc1))
    auto kc = [&](int d, int i, int c) {
        const double kk = (double)symid(i, G.symstart[d]) + G.koffset[d];
        return mkc((T)fd_symbol(G.odiff, kk * G.kfact[d][c][0], G.hgrid[d]), (T)fd_symbol(G.odiff, kk * G.kfact[d][c][1], G.hgrid[d]));
    };
    const C kx1 = kc(0, x, 1), kx2 = kc(0, x, 2), ky0 = kc(1, y, 0), ky2 = kc(1, y, 2);
    const T nf = (T)G.normfact;
    C* p0 = data + (3 * grp + 0) * A.cstr + oxy;
    C* p1 = data + (3 * grp + 1) * A.cstr + oxy;
    C* p2 = data + (3 * grp + 2) * A.cstr + oxy;
    for (int z = z0; z < z1; ++z) {
        const int64_t o = (int64_t)z * A.str[2];
        const C kz0 = kc(2, z, 0), kz1 = kc(2, z, 1);
        const T g = (T)green[gxy + (int64_t)gfold(z, G.gfold[2]) * G.gstr[2]] * nf;
        const C f0 = p0[o], f1 = p1[o], f2 = p2[o];
        const C r0 = csub(cmul(f2, ky2), cmul(f1, kz1));
        const C r1 = csub(cmul(f0, kz0), cmul(f2, kx2));
        const C r2 = csub(cmul(f1, kx1), cmul(f0, ky0));
        p0[o] = mkc(r0.x * g, r0.y * g);
        p1[o] = mkc(r1.x * g, r1.y * g);
        p2[o] = mkc(r2.x * g, r2.y * g);
    }
}

cudaError_t launch_spec_mult(const RotArgs& A, int data_f64, int green_f64, cudaStream_t s) {
    const int groups = (A.mult.mode == 2) ? A.nbatch : A.ncomp;
    if ((int64_t)A.n[0] * A.n[1] * A.n[2] * groups == 0) return cudaSuccess;
    const int zb = 32;
    const int nzc = (A.n[2] + zb - 1) / zb;
    if (A.n[1] > 65535 || (int64_t)nzc * groups > 65535) return cudaErrorInvalidValue;
    const dim3 grid((A.n[0] + 127) / 128, A.n[1], nzc * groups);
    if (data_f64 && green_f64) spec_mult_kernel<double, double><<<grid, 128, 0, s>>>(A, zb);
    else if (data_f64) spec_mult_kernel<double, float><<<grid, 128, 0, s>>>(A, zb);
    else spec_mult_kernel<float, float><<<grid, 128, 0, s>>>(A, zb);
    return cudaGetLastError();
}

// K_{d,c}(i) of the curl for every direction d, component c and spectral
// index i < n[d] (the values spec_mult_kernel forms per point), in the
// working precision: table (d, c) at out + (3 d + c) kstr
template <typename T>
__global__ void ksym_kernel(MultSpec G, int n0, int n1, int n2, int kstr, void* out) {
    using C = typename CT<T>::C;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 9 * kstr) return;
    const int d = e / (3 * kstr), c = (e / kstr) % 3, i = e % kstr;
    const int n = d == 0 ? n0 : (d == 1 ? n1 : n2);
    C k = mkc((T)0, (T)0);
    if (i < n) {
        const double kk = (double)symid(i, G.symstart[d]) + G.koffset[d];
        k = mkc((T)fd_symbol(G.odiff, kk * G.kfact[d][c][0], G.hgrid[d]), (T)fd_symbol(G.odiff, kk * G.kfact[d][c][1], G.hgrid[d]));
    }
    reinterpret_cast<C*>(out)[e] = k;
}

cudaError_t launch_ksym_table(const MultSpec& G, const int n[3], int kstr, void* out, int f64, cudaStream_t s) {
    const int tot = 9 * kstr;
    const int nb = (tot + 255) / 256;
    if (f64) ksym_kernel<double><<<nb, 256, 0, s>>>(G, n[0], n[1], n[2], kstr, out);
    else ksym_kernel<float><<<nb, 256, 0, s>>>(G, n[0], n[1], n[2], kstr, out);
    return cudaGetLastError();
}

}  // namespace flb
