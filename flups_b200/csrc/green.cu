// FP64 Green's function evaluation and finalisation kernels (see green.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <math_constants.h>

#include "green.cuh"
#include "lgf1unb.cuh"

namespace flb {

#define C_PI 3.14159265358979323846
#define C_1O4PI (1.0 / (4.0 * C_PI))
#define C_1O2PI (1.0 / (2.0 * C_PI))
#define C_1OPI (1.0 / C_PI)
#define C_1O2PI2 (1.0 / (2.0 * C_PI * C_PI))
#define C_1OSQRT2 0.70710678118654752440
#define C_1OSQRTPI 0.56418958354775628695
#define C_GAMMA 0.5772156649015328606

// ------------------------------------------------------------ special functions
__device__ __forceinline__ double horner(const double* c, int n, double x) {
    double a = c[n - 1];
    for (int i = n - 2; i >= 0; --i) a = a * x + c[i];
    return a;
}

// Numerical Recipes 3rd ed. sec. 6.5.1 rational approximations of K0 and K1
__device__ double besselk0_d(double x) {
    const double k0pi[5] = {1.0, 2.346487949187396e-1, 1.187082088663404e-2, 2.150707366040937e-4, 1.425433617130587e-6};
    const double k0qi[3] = {9.847324170755358e-1, 1.518396076767770e-2, 8.362215678646257e-5};
    const double k0p[5] = {1.159315156584126e-1, 2.770731240515333e-1, 2.066458134619875e-2, 4.574734709978264e-4,
                           3.454715527986737e-6};
    const double k0q[3] = {9.836249671709183e-1, 1.627693622304549e-2, 9.809660603621949e-5};
    const double k0pp[8] = {1.253314137315499, 1.475731032429900e1, 6.123767403223466e1, 1.121012633939949e2,
                            9.285288485892228e1, 3.198289277679660e1, 3.595376024148513, 6.160228690102976e-2};
    const double k0qq[8] = {1.0, 1.189963006673403e1, 5.027773590829784e1, 9.496513373427093e1, 8.318077493230258e1,
                            3.181399777449301e1, 4.443672926432041, 1.408295601966600e-1};
    if (x <= 1.0) {
        const double z = x * x;
        const double term = horner(k0pi, 5, z) * log(x) / horner(k0qi, 3, 1. - z);
        return horner(k0p, 5, z) / horner(k0q, 3, 1. - z) - term;
    }
    const double z = 1. / x;
    return exp(-x) * horner(k0pp, 8, z) / (horner(k0qq, 8, z) * sqrt(x));
}

__device__ double besselk1_d(double x) {
    const double k1pi[5] = {0.5, 5.598072040178741e-2, 1.818666382168295e-3, 2.397509908859959e-5, 1.239567816344855e-7};
    const double k1qi[3] = {9.870202601341150e-1, 1.292092053534579e-2, 5.881933053917096e-5};
    const double k1p[5] = {-3.079657578292062e-1, -8.109417631822442e-2, -3.477550948593604e-3, -5.385594871975406e-5,
                           -3.110372465429008e-7};
    const double k1q[3] = {9.861813171751389e-1, 1.375094061153160e-2, 6.774221332947002e-5};
    const double k1pp[8] = {1.253314137315502, 1.457171340220454e1, 6.063161173098803e1, 1.147386690867892e2,
                            1.040442011439181e2, 4.356596656837691e1, 7.265230396353690, 3.144418558991021e-1};
    const double k1qq[8] = {1.0, 1.125154514806458e1, 4.427488496597630e1, 7.616113213117645e1, 5.863377227890893e1,
                            1.850303673841586e1, 1.857244676566022, 2.538540887654872e-2};
    if (x <= 1.0) {
        const double z = x * x;
        const double term = horner(k1pi, 5, z) * log(x) / horner(k1qi, 3, 1. - z);
        return x * (horner(k1p, 5, z) / horner(k1q, 3, 1. - z) + term) + 1. / x;
    }
    const double z = 1.0 / x;
    return exp(-x) * horner(k1pp, 8, z) / (horner(k1qq, 8, z) * sqrt(x));
}

__device__ double clenshaw(const double* a, int n, double t) {
    double b0 = a[n - 1], b1 = 0.0, b2 = 0.0;
    for (int k = n - 2; k >= 0; --k) {
        b2 = b1;
        b1 = b0;
        b0 = t * b1 - b2 + a[k];
    }
    return 0.5 * (b0 - b2);
}

// E1 from two Chebyshev expansions ([-4,4] in x/4, [4,inf) in 4/x); 0 below -4
__device__ double expint_e1_d(double x) {
    const double a[23] = {7.8737715392882774, -8.0314874286705335, 3.8797325768522250, -1.6042971072992259,
                          0.5630905453891458, -0.1704423017433357, 0.0452099390015415, -0.0106538986439085,
                          0.0022562638123478, -0.0004335700473221, 0.0000762166811878, -0.0000123417443064,
                          0.0000018519745698, -0.0000002588698662, 0.0000000338604319, -0.0000000041611418,
                          0.0000000004821606, -0.0000000000528465, 0.0000000000054945, -0.0000000000005433,
                          0.0000000000000512, -0.0000000000000046, 0.0000000000000004};
    const double b[23] = {0.2155283776715125, 0.1028106215227030, -0.0045526707131788, 0.0003571613122851,
                          -0.0000379341616932, 0.0000049143944914, -0.0000007355024922, 0.0000001230603606,
                          -0.0000000225236907, 0.0000000044412375, -0.0000000009328509, 0.0000000002069297,
                          -0.0000000000481502, 0.0000000000116891, -0.0000000000029474, 0.0000000000007691,
                          -0.0000000000002070, 0.0000000000000573, -0.0000000000000163, 0.0000000000000047,
                          -0.0000000000000014, 0.0000000000000004, -0.0000000000000001};
    if (x >= -4. && x <= 4.) return -(clenshaw(a, 23, 2. * (.25 * x)) + log(fabs(x)));
    if (x > 4.) return clenshaw(b, 23, 2. * (2. * (4. / x) - 1.)) * exp(-x);
    return 0.0;
}

// Si(x) from the Chebyshev-Pade fits published with GalSim
__device__ double sine_integral_d(double x) {
    const double x2 = x * x;
    if (x2 > 16.) {
        const double y = 1. / x2;
        const double fn[11] = {1., 7.44437068161936700618e2, 1.96396372895146869801e5, 2.37750310125431834034e7,
                               1.43073403821274636888e9, 4.33736238870432522765e10, 6.40533830574022022911e11,
                               4.20968180571076940208e12, 1.00795182980368574617e13, 4.94816688199951963482e12,
                               -4.94701168645415959931e11};
        const double fd[11] = {1., 7.46437068161927678031e2, 1.97865247031583951450e5, 2.41535670165126845144e7,
                               1.47478952192985464958e9, 4.58595115847765779830e10, 7.08501308149515401563e11,
                               5.06084464593475076774e12, 1.43468549171581016479e13, 1.11535493509914254097e13, 0.};
        const double gn[11] = {1., 8.1359520115168615e2, 2.35239181626478200e5, 3.12557570795778731e7,
                               2.06297595146763354e9, 6.83052205423625007e10, 1.09049528450362786e12,
                               7.57664583257834349e12, 1.81004487464664575e13, 6.43291613143049485e12,
                               -1.36517137670871689e12};
        const double gd[11] = {1., 8.19595201151451564e2, 2.40036752835578777e5, 3.26026661647090822e7,
                               2.23355543278099360e9, 7.87465017341829930e10, 1.39866710696414565e12,
                               1.17164723371736605e13, 4.01839087307656620e13, 3.99653257887490811e13, 0.};
        const double f = horner(fn, 11, y) / (x * horner(fd, 10, y));
        const double g = y * horner(gn, 11, y) / horner(gd, 10, y);
        return ((x > 0.) ? (C_PI / 2.) : (-C_PI / 2.)) - f * cos(x) - g * sin(x);
    }
    const double pn[8] = {1., -4.54393409816329991e-2, 1.15457225751016682e-3, -1.41018536821330254e-5,
                          9.43280809438713025e-8, -3.53201978997168357e-10, 7.08240282274875911e-13, -6.05338212010422477e-16};
    const double pd[7] = {1., 1.01162145739225565e-2, 4.99175116169755106e-5, 1.55654986308745614e-7,
                          3.28067571055789734e-10, 4.5049097575386581e-13, 3.21107051193712168e-16};
    return x * horner(pn, 8, x2) / horner(pd, 7, x2);
}

// int_0^x (1 - J0(u))/u du, Humbert's series truncated at 50 terms (double precision here)
// double-double numbers (hi + lo, |lo| <= ulp(hi) / 2): error-free sums
// (Knuth's two-sum) and products (an FMA gives the rounding error of hi * hi)
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD dd_norm(double s, double e) {
    const double hi = __dadd_rn(s, e);
    return {hi, __dadd_rn(e, -__dadd_rn(hi, -s))};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
    const double s = __dadd_rn(a.hi, b.hi);
    const double bb = __dadd_rn(s, -a.hi);
    const double e = __dadd_rn(__dadd_rn(a.hi, -__dadd_rn(s, -bb)), __dadd_rn(b.hi, -bb));
    return dd_norm(s, __dadd_rn(e, __dadd_rn(a.lo, b.lo)));
}
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    const double p = __dmul_rn(a.hi, b.hi);
    const double e = __fma_rn(a.hi, b.hi, -p);
    return dd_norm(p, __dadd_rn(e, __dadd_rn(__dmul_rn(a.hi, b.lo), __dmul_rn(a.lo, b.hi))));
}
__device__ __forceinline__ DD dd_div(DD a, double b) {
    const double q1 = __ddiv_rn(a.hi, b);
    const DD r = dd_add(a, {-__dmul_rn(q1, b), -__fma_rn(q1, b, -__dmul_rn(q1, b))});
    return dd_norm(q1, __ddiv_rn(r.hi, b));
}

// The same truncated series as the reference (50 terms of Humbert's
// expansion, src/ji0.hpp:37-44), summed in double-double: its alternating
// terms reach 1e11 at x = 30 against a sum of about 3, which leaves a double
// sum a relative error of 1e-5 there (the reference's long double, 1e-9)
__device__ double ji0c_d(double x) {
    const DD q = dd_mul({-0.25, 0.0}, dd_mul({x, 0.0}, {x, 0.0}));
    DD t = {1.0, 0.0}, val = {0.0, 0.0};
    for (int n = 1; n <= 50; ++n) {
        t = dd_div(dd_mul(t, q), (double)n * (double)n);  // q^n / (n!)^2
        const DD u = dd_div(t, 2.0 * n);
        val = dd_add(val, {-u.hi, -u.lo});
    }
    return __dadd_rn(val.hi, val.lo);
}

__device__ __forceinline__ double lgf2_symbol(double k) {
    const double s = sin(k / 2.);
    return 4.0 * s * s;
}
__device__ __forceinline__ double lgf4_symbol(double k) {
    const double s = sin(k / 2.), t = sin(k);
    return 4.0 * (4. / 3. * s * s - 1. / 12. * t * t);
}
__device__ __forceinline__ double lgf6_symbol(double k) {
    const double s = sin(k / 2.), t = sin(k), u = sin(1.5 * k);
    return 4.0 * (3. / 2. * s * s - 3. / 20. * t * t + 1. / 90. * u * u);
}
__device__ __forceinline__ double lgf8_symbol(double k) {
    const double s = sin(k / 2.), t = sin(k), u = sin(1.5 * k), v = sin(2. * k);
    return 4.0 * (8. / 5. * s * s - 1. / 5. * t * t + 8. / 315. * u * u - 1. / 560. * v * v);
}

// closed-form 1-D LGF of the 3-point stencil with a spectral shift c >= 0
__device__ double lgf2_1unb_d(int n, double c) {
    n = abs(n);
    if (c == 0.0) return -0.5 * n;
    if (c < 1.0e-3) {
        const double rm1 = c / 2. - sqrt(c * c / 4. + c);
        double ls = 0.0, vm = 0.0;
        for (int i = 0; i < 12; ++i) {
            ls += 1.0 / (12 - i);
            ls *= -rm1;
            vm += 1.0;
            vm *= -rm1;
        }
        ls = -ls;
        vm = -vm + rm1;
        return -exp(n * ls) / vm;
    }
    const double r = 1 + c / 2. - sqrt(c * c / 4. + c);
    return -pow(r, (double)n) / (r - 1. / r);
}

__device__ __forceinline__ double ipow(double x, int e) {
    if (e == 0) return 1.0;
    bool neg = e < 0;
    unsigned u = neg ? (unsigned)(-e) : (unsigned)e;
    double r = 1.0, b = x;
    while (u) {
        if (u & 1u) r *= b;
        b *= b;
        u >>= 1;
    }
    return neg ? 1.0 / r : r;
}

__device__ double farfield_eval(const GreenEvalArgs& A, double n1, double n2, double n3) {
    const double n = sqrt(n1 * n1 + n2 * n2 + n3 * n3);
    double s = 0.0;
    for (int t = 0; t < A.nfar; ++t) {
        const FarTerm f = A.far[t];
        s += f.coef * ipow(n1, f.a) * ipow(n2, f.b) * ipow(n3, f.c) * ipow(n, f.e);
    }
    if (A.far_log != 0.0) s += A.far_log * log(n);
    return s;
}

__device__ __forceinline__ bool is_hej(int k) { return k == G_HEJ_2 || k == G_HEJ_4 || k == G_HEJ_6 || k == G_HEJ_8 || k == G_HEJ_10; }
__device__ __forceinline__ bool is_lgf_or_mehr(int k) {
    return k == G_LGF_2 || k == G_LGF_4 || k == G_LGF_6 || k == G_LGF_8 || k == G_MEHR_4L || k == G_MEHR_6L ||
           k == G_MEHR_4F || k == G_MEHR_6F;
}

// ------------------------------------------------------------ kernels per splitting
__device__ double g_3unb(const GreenEvalArgs& A, double r, int i0, int i1, int i2) {
    const double eps = A.length;
    const int k = A.kind;
    if (is_lgf_or_mehr(k)) {
        const int N = A.tableN;
        double g;
        if (i0 < N && i1 < N && i2 < N) g = A.table[i0 + i1 * N + i2 * N * N];
        else g = farfield_eval(A, (double)i0, (double)i1, (double)i2);
        return -g / A.hgrid;
    }
    const double rho = r / eps;
    const double ex = exp(-rho * rho * .5);
    const double ef = erf(rho * C_1OSQRT2);
    const double pre = C_1OSQRT2 * C_1OSQRTPI;
    switch (k) {
        case G_HEJ_2: return -C_1O4PI / r * erf(r / eps * C_1OSQRT2);
        case G_HEJ_4: return -C_1O4PI / r * (pre * rho * ex + ef);
        case G_HEJ_6: return -C_1O4PI / r * (pre * (7. / 4. * rho - 1. / 4. * rho * rho * rho) * ex + ef);
        case G_HEJ_8: {
            const double r3 = rho * rho * rho, r5 = r3 * rho * rho;
            return -C_1O4PI / r * (pre * (19. / 8 * rho - 2. / 3 * r3 + 1. / 24 * r5) * ex + ef);
        }
        case G_HEJ_10: {
            const double r3 = rho * rho * rho, r5 = r3 * rho * rho, r7 = r5 * rho * rho;
            return -C_1O4PI / r * (pre * (187. / 64. * rho - 233. / 192. * r3 + 29. / 192. * r5 - 1. / 192. * r7) * ex + ef);
        }
        case G_HEJ_0: return -C_1O2PI2 * (1.0 / eps) * sine_integral_d(rho) / rho;
        case G_CHAT_2: return -C_1O4PI / r;
    }
    return 0.0;
}

__device__ double g_2d_table(const GreenEvalArgs& A, int ix, int iy, int iz) {
    const int i1 = (ix == 0) ? iy : ix;
    const int i2 = (ix == 0) ? iz : ((iy == 0) ? iz : iy);
    const int N = A.tableN;
    double g;
    if (i1 < N && i2 < N) g = A.table[i1 + i2 * N];
    else g = farfield_eval(A, (double)i1, (double)i2, 0.0);
    return -g;
}

__device__ double g_2unb1spe(const GreenEvalArgs& A, double r, double k, int i0, int i1, int i2) {
    const int kind = A.kind;
    const double sig = A.length;
    const bool r0 = r <= A.r_cut;
    const bool k0 = !r0 && (k <= A.k_cut);
    if (is_lgf_or_mehr(kind)) return (r0 || k0) ? g_2d_table(A, i0, i1, i2) : 0.0;
    if (is_hej(kind)) {
        if (!(r0 || k0)) return 0.0;
        double poly_c = 0.0;
        if (kind == G_HEJ_4) poly_c = 0.5;
        else if (kind == G_HEJ_6) poly_c = 0.75;
        else if (kind == G_HEJ_8) poly_c = 11. / 12.;
        else if (kind == G_HEJ_10) poly_c = 25. / 24.;
        if (r0) return -C_1O2PI * (C_GAMMA * .5 - log(1.41421356237309504880 * sig) + poly_c);
        const double rho2 = (r / sig) * (r / sig);
        double poly = 0.0;
        if (kind == G_HEJ_4) poly = 0.5;
        else if (kind == G_HEJ_6) poly = 0.75 - 0.125 * rho2;
        else if (kind == G_HEJ_8) poly = 11. / 12. - 7. / 24. * rho2 + 1. / 48. * rho2 * rho2;
        else if (kind == G_HEJ_10) poly = 25. / 24. - 23. / 48. * rho2 + 13. / 192. * rho2 * rho2 - 1. / 384. * rho2 * rho2 * rho2;
        if (kind == G_HEJ_2) return C_1O2PI * (log(r) + 0.5 * expint_e1_d(rho2 * 0.5));
        return C_1O2PI * (log(r) - poly * exp(-rho2 * 0.5) + 0.5 * expint_e1_d(rho2 * 0.5));
    }
    if (kind == G_HEJ_0) {
        if (!(r0 || k0)) return 0.0;
        const double rho = r / sig;
        const double tmp = C_1O2PI * (ji0c_d(rho) + log(2 * sig) - C_GAMMA);
        return (rho < 30.0) ? tmp : C_1O2PI * log(r);
    }
    // CHAT_2
    if (r0) {
        const double kr = k * A.r_eq2d;
        return -(1.0 - kr * besselk1_d(kr)) * C_1OPI / (kr * kr);
    }
    if (k0) return C_1O2PI * log(r);
    return -C_1O2PI * besselk0_d(fabs(k) * r);
}

// 1 - erf(x) as the reference forms it (src/green_kernels.hpp:469): 1 minus
// the double nearest erf(x).
// For x >= 2, 1 - erfc(x) rounds to that double (erfc(x) < 0.005 is known
// far below half an ulp of 1) and the subtraction from 1 is exact, whereas
// erf(x) itself may come out an ulp away; hej_1unb multiplies the result by
// exp(s rho), which turns that ulp into a relative error of up to 1e-4 in a
// Green's value (and 1e-12 - 1e-11 in a solve)
__device__ double one_minus_erf(double x) {
    if (x >= 2.0) return __dadd_rn(1.0, -__dadd_rn(1.0, -erfc(x)));
    return 1.0 - erf(x);
}

__device__ double hej_1unb(int kind, double r, double k, double sig, bool zero_k) {
    const double rho = r / sig;
    const double rosqrt2 = r * C_1OSQRT2;
    const double er = exp(-rho * rho * .5);
    const double q = sig * C_1OSQRT2 * C_1OSQRTPI;
    if (zero_k) {
        const double base = 0.5 * r * erf(rosqrt2 / sig);
        const double rho2 = rho * rho;
        switch (kind) {
            case G_HEJ_2: return base - (1. - er) * q;
            case G_HEJ_4: return base - (1. - er) * .5 * q;
            case G_HEJ_6: return base - (3. - er * (rho2 + 3.)) * .125 * q;
            case G_HEJ_8: return base - (5. / 16. - er * (-1. / 48. * rho2 * rho2 + .25 * rho2 + 5. / 16.)) * q;
            default:
                return base - (35. / 128. - er * (1. / 384. * rho2 * rho2 * rho2 - 23. / 384. * rho2 * rho2 + 47. / 128. * rho2 +
                                                  35. / 128.)) * q;
        }
    }
    const double s = k * sig;
    const double s2 = s * s, rho2 = rho * rho;
    const double sub = (s * rho > 100.) ? 0.0
                                        : (one_minus_erf(C_1OSQRT2 * (s - rho)) * exp(-s * rho) +
                                           one_minus_erf(C_1OSQRT2 * (s + rho)) * exp(s * rho));
    const double base = -.25 * sig / s * sub;
    const double pre = sig * 1.41421356237309504880 * C_1OSQRTPI;
    const double e = exp(-.5 * (s * s + rho * rho));
    switch (kind) {
        case G_HEJ_2: return base;
        case G_HEJ_4: return base - pre * .25 * e;
        case G_HEJ_6: return base - pre * (5. / 16. + 1. / 16. * (s2 - rho2)) * e;
        case G_HEJ_8:
            return base - pre * (11. / 32. + 1. / 12. * s2 - 0.125 * rho2 - 1. / 48. * s2 * rho2 + 1. / 96. * (s2 * s2 + rho2 * rho2)) * e;
        default:
            return base - pre * (93. / 256. + 73. / 768. * s2 - 47. / 256. * rho2 - 17. / 384. * s2 * rho2 + 11. / 768. * s2 * s2 +
                                 23. / 768. * rho2 * rho2 + 1. / 256. * (s2 * rho2 * rho2 - s2 * s2 * rho2) +
                                 1. / 768. * (s2 * s2 * s2 - rho2 * rho2 * rho2)) * e;
    }
}

__device__ double g_1unb2spe(const GreenEvalArgs& A, double r, double k, double ka, double kb, double kc) {
    const int kind = A.kind;
    const bool zk = k <= A.k_cut;
    if (is_hej(kind)) return hej_1unb(kind, r, k, A.length, zk);
    if (kind == G_CHAT_2) return zk ? 0.5 * fabs(r) : -0.5 * exp(-k * r) / k;
    const double h = A.hgrid;
    const int n = (int)round(fabs(r) / h);
    switch (kind) {
        case G_LGF_2: return -h * lgf2_1unb_d(n, lgf2_symbol(ka * h) + lgf2_symbol(kb * h) + lgf2_symbol(kc * h));
        case G_LGF_4: return -h * lgf1::lgf4(n, lgf4_symbol(ka * h) + lgf4_symbol(kb * h) + lgf4_symbol(kc * h));
        case G_LGF_6: return -h * lgf1::lgf6(n, lgf6_symbol(ka * h) + lgf6_symbol(kb * h) + lgf6_symbol(kc * h));
        case G_LGF_8: return -h * lgf1::lgf8(n, lgf8_symbol(ka * h) + lgf8_symbol(kb * h) + lgf8_symbol(kc * h));
    }
    // Mehrstellen: one of the wave numbers is zero; |k1| >= |k2| >= 0
    const double k1 = fmax(fabs(ka), fmax(fabs(kb), fabs(kc)));
    const double k2 = fabs(ka) + fabs(kb) + fabs(kc) - k1;
    switch (kind) {
        case G_MEHR_4L: return -h * lgf1::meh4(n, k1 * h, k2 * h, false);
        case G_MEHR_4F: return -h * lgf1::meh4(n, k1 * h, k2 * h, true);
        case G_MEHR_6L: return -h * lgf1::meh6(n, k1 * h, k2 * h, false);
        case G_MEHR_6F: return -h * lgf1::meh6(n, k1 * h, k2 * h, true);
    }
    return 0.0;  // not reached: HEJ_0 is refused by the host in this splitting
}

__device__ double g_0unb3spe(int kind, double ksqr, double k0, double k1, double k2, double h, double sig) {
    const double s = ksqr * (sig * sig);
    const double e = exp(-s * 0.5);
    switch (kind) {
        case G_HEJ_2: return -e / ksqr;
        case G_HEJ_4: return -(1.0 + s * 0.5) * e / ksqr;
        case G_HEJ_6: return -(1.0 + s * 0.5 + s * s * 0.125) * e / ksqr;
        case G_HEJ_8: { const double s2 = s * s; return -(1.0 + s * 0.5 + s2 * 0.125 + s2 * s * (1. / 48.)) * e / ksqr; }
        case G_HEJ_10: {
            const double s2 = s * s;
            return -(1.0 + s * 0.5 + s2 * 0.125 + s2 * s * (1. / 48.) + s2 * s2 * (1. / 384.)) * e / ksqr;
        }
        case G_CHAT_2:
        case G_HEJ_0: return -1.0 / ksqr;
        case G_LGF_2: return -h * h / (lgf2_symbol(k0 * h) + lgf2_symbol(k1 * h) + lgf2_symbol(k2 * h));
        case G_LGF_4: return -h * h / (lgf4_symbol(k0 * h) + lgf4_symbol(k1 * h) + lgf4_symbol(k2 * h));
        case G_LGF_6: return -h * h / (lgf6_symbol(k0 * h) + lgf6_symbol(k1 * h) + lgf6_symbol(k2 * h));
        case G_LGF_8: return -h * h / (lgf8_symbol(k0 * h) + lgf8_symbol(k1 * h) + lgf8_symbol(k2 * h));
        default: break;
    }
    const double y0 = sin(k0 * h / 2.) * sin(k0 * h / 2.);
    const double y1 = sin(k1 * h / 2.) * sin(k1 * h / 2.);
    const double y2 = sin(k2 * h / 2.) * sin(k2 * h / 2.);
    double left = -4. * (y0 + y1 + y2) + 8. / 3. * (y0 * y1 + y1 * y2 + y0 * y2);
    if (kind == G_MEHR_6L || kind == G_MEHR_6F) left -= 32. / 15. * y0 * y1 * y2;
    if (kind == G_MEHR_4L || kind == G_MEHR_6L) return h * h / left;
    if (kind == G_MEHR_4F) return h * h * (1. - 1. / 3. * (y0 + y1 + y2)) / left;
    const double right = 1. - 1. / 3. * (y0 + y1 + y2) + 8. / 45. * (y0 * y1 + y1 * y2 + y0 * y2) -
                         1. / 15. * (y0 * y0 + y1 * y1 + y2 * y2);
    return h * h * right / left;
}

__device__ __forceinline__ int symid_g(int i, double symstart) {
    if (symstart == 0.0 || (double)i <= symstart) return i;
    int a = (int)fabs(2.0 * symstart - (double)i);
    return -(a > 1 ? a : 1);
}

__global__ void green_eval_kernel(const GreenEvalArgs A) {
    const int64_t n0 = A.size[0], n1 = A.size[1];
    const int64_t c0 = A.canon ? A.csize[0] : A.size[0], c1 = A.canon ? A.csize[1] : A.size[1];
    const int64_t c2 = A.canon ? A.csize[2] : A.size[2];
    const int64_t total = c0 * c1 * c2;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int I[3];
        I[0] = (int)(t % c0);
        I[1] = (int)((t / c0) % c1);
        I[2] = (int)(t / (c0 * c1));
        const int64_t id = I[0] + n0 * (I[1] + n1 * (int64_t)I[2]);
        int is[3];
        double x[3], kk[3];
        for (int d = 0; d < 3; ++d) {
            is[d] = symid_g(I[d], A.symstart[d]);
            x[d] = is[d] * A.hfact[d];
            kk[d] = (is[d] + A.koffset[d]) * A.kfact[d];
        }
        const int a0 = abs(is[A.ax[0]]), a1 = abs(is[A.ax[1]]), a2 = abs(is[A.ax[2]]);
        double g = 0.0;
        if (A.nunb == 3) {
            const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
            g = g_3unb(A, r, a0, a1, a2);
            if (A.set_g0 && id == 0) g = A.g0;
        } else if (A.nunb == 2) {
            const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
            const double k = kk[0] + kk[1] + kk[2];
            g = g_2unb1spe(A, r, k, a0, a1, a2);
            if (A.chat2d_origin && id == 0)
                g = 0.25 * C_1O2PI * (C_PI - 6.0 + 2.0 * log(0.5 * C_PI * A.r_eq2d * A.r_eq2d));
        } else if (A.nunb == 1) {
            const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
            const double k = sqrt(kk[0] * kk[0] + kk[1] * kk[1] + kk[2] * kk[2]);
            g = g_1unb2spe(A, r, k, kk[A.ax[0]], kk[A.ax[1]], kk[A.ax[2]]);
        } else {
            const double ksqr = kk[0] * kk[0] + kk[1] * kk[1] + kk[2] * kk[2];
            g = g_0unb3spe(A.kind, ksqr, kk[A.ax[0]], kk[A.ax[1]], kk[A.ax[2]], A.hgrid, A.length);
            if (A.set_g0 && id == 0) g = 0.0;
        }
        if (A.cplx) {
            A.out[2 * id] = g;
            A.out[2 * id + 1] = 0.0;
        } else {
            A.out[id] = g;
        }
    }
}

// every index outside the canonical box takes the value of its mirror image
// |symid| inside the box (3 unbounded directions: the function depends on |is|)
__global__ void green_mirror_kernel(const GreenEvalArgs A) {
    const int64_t n0 = A.size[0], n1 = A.size[1], n2 = A.size[2];
    const int64_t total = n0 * n1 * n2;
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < total; id += (int64_t)gridDim.x * blockDim.x) {
        int I[3], S[3];
        I[0] = (int)(id % n0);
        I[1] = (int)((id / n0) % n1);
        I[2] = (int)(id / (n0 * n1));
        bool inside = true;
        for (int d = 0; d < 3; ++d) {
            S[d] = I[d] < A.csize[d] ? I[d] : abs(symid_g(I[d], A.symstart[d]));
            inside = inside && (I[d] < A.csize[d]);
        }
        if (inside) continue;
        const int64_t src = S[0] + n0 * (S[1] + n1 * (int64_t)S[2]);
        if (A.cplx) {
            A.out[2 * id] = A.out[2 * src];
            A.out[2 * id + 1] = 0.0;
        } else {
            A.out[id] = A.out[src];
        }
    }
}

__global__ void green_final_kernel(const GreenFinalArgs A) {
    const int64_t n0 = A.fold_n[0], n1 = A.fold_n[1], n2 = A.fold_n[2];
    const int64_t total = n0 * n1 * n2;
    const int64_t s0 = A.spec_n[0], s1 = A.spec_n[1];
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < total; id += (int64_t)gridDim.x * blockDim.x) {
        int I[3];
        I[0] = (int)(id % n0);
        I[1] = (int)((id / n0) % n1);
        I[2] = (int)(id / (n0 * n1));
        const int64_t src = I[0] + s0 * (I[1] + s1 * (int64_t)I[2]);
        double v = (A.spec_cplx ? A.spec[2 * src] : A.spec[src]) * A.volfact;
        if (A.complete && I[A.spec_dim] >= 1) {
            double kk[3];
            for (int d = 0; d < 3; ++d) kk[d] = (symid_g(I[d], A.symstart[d]) + A.koffset[d]) * A.kfact[d];
            const double ksqr = kk[0] * kk[0] + kk[1] * kk[1] + kk[2] * kk[2];
            v = g_0unb3spe(A.kind, ksqr, kk[A.ax[0]], kk[A.ax[1]], kk[A.ax[2]], A.hgrid, A.length);
        }
        if (A.reset0 && id == 0) v = 0.0;
        v *= A.scale;
        const int64_t o = I[0] * A.fold_str[0] + I[1] * A.fold_str[1] + I[2] * A.fold_str[2];
        if (A.out_f64) reinterpret_cast<double*>(A.out)[o] = v;
        else reinterpret_cast<float*>(A.out)[o] = (float)v;
    }
}

cudaError_t launch_green_eval(const GreenEvalArgs& Ain, cudaStream_t s) {
    GreenEvalArgs A = Ain;
    A.canon = 0;
    if (A.nunb == 3) {
        // the canonical box: 0..floor(symstart) along each mirrored direction;
        // beyond it |symid| falls back inside the box
        A.canon = 1;
        for (int d = 0; d < 3; ++d) {
            int c = A.size[d];
            if (A.symstart[d] > 0.0) c = std::min(A.size[d], (int)floor(A.symstart[d]) + 1);
            A.csize[d] = c;
        }
    }
    const int64_t total = A.canon ? (int64_t)A.csize[0] * A.csize[1] * A.csize[2] : (int64_t)A.size[0] * A.size[1] * A.size[2];
    int64_t nb = (total + 255) / 256;
    if (nb > 148 * 64) nb = 148 * 64;
    if (nb < 1) nb = 1;
    green_eval_kernel<<<(unsigned)nb, 256, 0, s>>>(A);
    if (A.canon) {
        const int64_t all = (int64_t)A.size[0] * A.size[1] * A.size[2];
        int64_t nm = (all + 255) / 256;
        if (nm > 148 * 64) nm = 148 * 64;
        green_mirror_kernel<<<(unsigned)std::max<int64_t>(nm, 1), 256, 0, s>>>(A);
    }
    return cudaGetLastError();
}

cudaError_t launch_green_final(const GreenFinalArgs& A, cudaStream_t s) {
    const int64_t total = (int64_t)A.fold_n[0] * A.fold_n[1] * A.fold_n[2];
    int64_t nb = (total + 255) / 256;
    if (nb > 148 * 64) nb = 148 * 64;
    if (nb < 1) nb = 1;
    green_final_kernel<<<(unsigned)nb, 256, 0, s>>>(A);
    return cudaGetLastError();
}

}  // namespace flb
