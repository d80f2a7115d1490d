// 1-D lattice Green's functions of one unbounded direction with the two
// other directions spectral (FP64, device; set-up only).
//
// With two spectral directions the lattice Poisson problem becomes, per
// wave-number pair, a 1-D problem A G = delta_n for the scheme's 1-D stencil
// A shifted by the symbol c of the spectral directions.  G(n) is a residue
// sum over the roots r (|r| < 1) of the stencil's characteristic polynomial;
// each regime of c (zero, small, real roots, a repeated root, complex roots)
// has its own closed form, restated from the reference's
// src/lgf_1unb2spe.hpp:161-612 (LGF2/4/6/8 and the Mehrstellen schemes,
// which take the two wave numbers instead of c).  The constants are the
// ones of those closed forms (series of the root nearest 1, residues at the
// repeated roots, the c = 0 forms).
#pragma once
#include <cuda_runtime.h>

namespace flb {
namespace lgf1 {

// ---------------------------------------------------------------- FP64 complex
struct zc {
    double x, y;
};
__device__ __forceinline__ zc Z(double a, double b = 0.0) { return zc{a, b}; }
__device__ __forceinline__ zc operator+(zc a, zc b) { return Z(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ zc operator-(zc a, zc b) { return Z(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ zc operator*(zc a, zc b) { return Z(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ zc operator*(double s, zc a) { return Z(s * a.x, s * a.y); }
__device__ __forceinline__ zc operator*(zc a, double s) { return Z(s * a.x, s * a.y); }
__device__ __forceinline__ zc operator+(zc a, double s) { return Z(a.x + s, a.y); }
__device__ __forceinline__ zc operator+(double s, zc a) { return Z(a.x + s, a.y); }
__device__ __forceinline__ zc operator-(zc a, double s) { return Z(a.x - s, a.y); }
__device__ __forceinline__ zc operator-(double s, zc a) { return Z(s - a.x, -a.y); }
// Smith's division
__device__ __forceinline__ zc operator/(zc a, zc b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, d = b.x + b.y * r;
        return Z((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    const double r = b.x / b.y, d = b.x * r + b.y;
    return Z((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ zc operator/(double s, zc b) { return Z(s) / b; }
__device__ __forceinline__ zc operator/(zc a, double s) { return Z(a.x / s, a.y / s); }
__device__ __forceinline__ zc conj(zc a) { return Z(a.x, -a.y); }
__device__ __forceinline__ double zabs(zc a) { return hypot(a.x, a.y); }
__device__ __forceinline__ double zarg(zc a) { return atan2(a.y, a.x); }
__device__ __forceinline__ double znorm(zc a) { return a.x * a.x + a.y * a.y; }
// principal square root (branch cut on the negative real axis, the sign of a
// zero imaginary part picks the side)
__device__ __forceinline__ zc zsqrt(zc a) {
    if (a.x == 0.0 && a.y == 0.0) return Z(0.0, a.y);
    const double t = sqrt(0.5 * (fabs(a.x) + hypot(a.x, a.y)));
    if (a.x >= 0.0) return Z(t, a.y / (2.0 * t));
    return Z(fabs(a.y) / (2.0 * t), copysign(t, a.y));
}
// z^e for a real exponent: the real power for a positive real z, else exp(e log z)
__device__ __forceinline__ zc zpow(zc a, double e) {
    if (a.y == 0.0 && a.x > 0.0) return Z(pow(a.x, e));
    const double lr = log(zabs(a)), th = zarg(a);
    const double m = exp(e * lr);
    double s, c;
    sincos(e * th, &s, &c);
    return Z(m * c, m * s);
}

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ double horn(const double* a, int n, double x) {
    double out = a[n - 1];
    for (int i = 2; i <= n; ++i) out = x * out + a[n - i];
    return out;
}
// log(x) and x - 1/x about x = 1, from x - 1
__device__ __forceinline__ double log_series(double xm1) {
    double out = 0.0;
    for (int i = 0; i < 12; ++i) {
        out += 1.0 / (12 - i);
        out *= -xm1;
    }
    return -out;
}
__device__ __forceinline__ double vmi_series(double xm1) {
    double out = 0.0;
    for (int i = 0; i < 12; ++i) {
        out += 1.0;
        out *= -xm1;
    }
    return -out + xm1;
}
// r = lambda - sqrt(lambda^2 - 1), |r| <= 1, also for large or infinite lambda
__device__ __forceinline__ double r_from_lambda(double lam) {
    if (isinf(lam)) return 0.0;
    if (fabs(lam) > 1.0e2) {
        const double e[10] = {0, 1. / 2., 0, 1. / 8., 0, 1. / 16., 0, 5. / 128., 0, 7. / 256.};
        return horn(e, 10, 1.0 / lam);
    }
    return (Z(lam) - zsqrt(Z(lam - 1)) * zsqrt(Z(lam + 1))).x;
}
// contribution of a conjugate root pair (root r, residue factor pp, stencil half-width w)
__device__ __forceinline__ double oscillatory(zc r, zc pp, int w, int n) {
    const zc K = Z(0.0, 2.0) * zpow(r, (double)(w - 1)) / pp;
    const int an = abs(n);
    return zabs(K) * pow(zabs(r), (double)an) * sin(zarg(r) * an + zarg(K));
}
// the real root nearest 1 for small c, from its series in c: r1 - 1
__device__ __forceinline__ double small_root_m1(const double* ser, double c) {
    const double lm1 = horn(ser, 8, c);
    return lm1 - sqrt(lm1 * lm1 + 2 * lm1);
}

// ---------------------------------------------------------------- symbols and stencil factors
__device__ __forceinline__ double sq(double v) { return v * v; }
__device__ __forceinline__ double sym4(double k) { return 4.0 * (4. / 3. * sq(sin(k / 2.)) - 1. / 12. * sq(sin(k))); }
__device__ __forceinline__ double sym6(double k) {
    return 4.0 * (3. / 2. * sq(sin(k / 2.)) - 3. / 20. * sq(sin(k)) + 1. / 90. * sq(sin(1.5 * k)));
}
__device__ __forceinline__ double sym8(double k) {
    return 4.0 * (8. / 5. * sq(sin(k / 2.)) - 1. / 5. * sq(sin(k)) + 8. / 315. * sq(sin(1.5 * k)) - 1. / 560. * sq(sin(2. * k)));
}
template <typename U>
__device__ __forceinline__ U pp4(U z, double c) { return -4. / 3. + z * ((5. + 2. * c) + z * (-4. + z / 3.)); }
template <typename U>
__device__ __forceinline__ U pp6(U z, double c) {
    return 3. / 20. + z * (-3. + z * ((49. / 6. + 3. * c) + z * (-6. + z * (3. / 4. - z / 15.))));
}
template <typename U>
__device__ __forceinline__ U pp8(U z, double c) {
    return -8. / 315. + z * (2. / 5. + z * (-24. / 5. + z * (205. / 18. + 4. * c + z * (-8. + z * (6. / 5. + z * (-8. / 45. + z / 70.))))));
}

// ---------------------------------------------------------------- LGF4 (5-point stencil)
__device__ inline double lgf4(int n, double c) {
    const int an = abs(n);
    if (c == 0.0) return -0.5 * an + -7.216878364870408e-2 * (pow(7.179676972449123e-2, (double)an) - 1.0);
    if (c < 1e-3) {
        const double ser[8] = {0, 0.5, 1. / 24., 1. / 144., 5. / 3456., 7. / 20736., 7. / 82944., 11. / 497664.};
        const double rm1 = small_root_m1(ser, c), r1 = rm1 + 1.0;
        const double lam2 = 4.0 + sqrt(9.0 - 3.0 * c);
        const double r2 = lam2 - sqrt(lam2 * lam2 - 1.0);
        const double pp1 = 1. / 12. * vmi_series(rm1) * (r1 - r2) * (r1 - 1.0 / r2);
        const double pp2 = pp4(r2, c);
        return exp((an + 1) * log_series(rm1)) / pp1 + pow(r2, (double)(an + 1)) / pp2;
    }
    if (c < 3.0 - 1e-5) {
        const double lam1 = 4.0 + sqrt(9.0 - 3.0 * c), lam2 = 4.0 - sqrt(9.0 - 3.0 * c);
        const double r1 = lam1 - sqrt(lam1 * lam1 - 1.0), r2 = lam2 - sqrt(lam2 * lam2 - 1.0);
        const double f1 = 12 * pow(r1, (double)(an + 1)) / ((r1 - 1.0 / r1) * (r1 - 1.0 / r2));
        const double f2 = 12 * pow(r2, (double)(an + 1)) / ((r2 - 1.0 / r1) * (r2 - 1.0 / r2));
        return (f1 - f2) / (r1 - r2);
    }
    if (c < 3.0 + 1e-5) {
        const double s15 = sqrt(15.);
        const double g0[2] = {4. / (5. * s15), 1. / 5.};
        const double g1[4] = {-14. / (75. * s15), -2. / 25., -4. / (25. * s15), -1. / 150.};
        const double g2[6] = {901. / (18750. * s15), 74. / 3125., 253. / (3750. * s15), 23. / 3750., 1. / (250. * s15), 1. / 15000.};
        const double g3[8] = {-37313. / (2812500. * s15), -11267. / 1640625., -3167. / (140625. * s15), -1. / 375.,
                              -31. / (11250. * s15), -31. / 281250., -1. / (28125. * s15), -1. / 3150000.};
        const double g4[10] = {3885631. / (1012500000. * s15), 1194829. / 590625000., 1118351. / (157500000. * s15),
                               12571. / 13125000., 13751. / (11250000. * s15), 127. / 1875000., 247. / (6750000. * s15),
                               13. / 15750000., 1. / (6300000. * s15), 1. / 1134000000.};
        const double nr = (double)an;
        const double g[5] = {horn(g0, 2, nr), horn(g1, 4, nr), horn(g2, 6, nr), horn(g3, 8, nr), horn(g4, 10, nr)};
        return pow(4.0 - s15, (double)an) * horn(g, 5, c - 3.0);
    }
    const zc lam = 4.0 - zsqrt(Z(9.0 - 3.0 * c));
    const zc r = lam - zsqrt(lam * lam - 1.0);
    const zc pp = Z(0.0, 1.0) / 6. * r.y * (r - 1. / r) * (r - 1. / conj(r));
    return oscillatory(r, pp, 2, n);
}

// ---------------------------------------------------------------- LGF6 (7-point stencil)
__device__ inline void lgf6_roots(double c, double& r1, zc& r2) {
    const double xi = cbrt(360. * c - 775. + 60. * sqrt(36. * c * c - 155. * c + 405.));
    const double lam1 = 0.25 * (9. - 95. / xi + xi);
    r1 = lam1 - sqrt(lam1 * lam1 - 1.0);
    const zc w = Z(-0.5, sqrt(3.) / 2.);
    const zc lam2 = 0.25 * (9. - 95. / (w * xi) + (w * xi));
    r2 = lam2 - zsqrt(lam2 * lam2 - 1.0);
}

__device__ inline double lgf6(int n, double c) {
    const int an = abs(n);
    if (c == 0.0) {
        const double a = 1.035017642406219e-1, p = 9.54295097909627e-2, t = -9.958762687216868e-1, f = -2.168575565241744e+0;
        return -0.5 * an + a * pow(p, (double)an) * sin(an * t + f) - a * sin(f);
    }
    double r1;
    zc r2;
    lgf6_roots(c, r1, r2);
    const zc p2 = pp6(r2, c);
    if (c < 1e-3) {
        const double ser[8] = {0, 0.5, 1. / 24., 1. / 720., -1. / 1152., -149. / 518400., -259. / 6220800., 163. / 62208000.};
        const double rm1 = small_root_m1(ser, c), q1 = rm1 + 1.0;
        const double pp1 = -1. / 90. * vmi_series(rm1) * znorm((q1 - r2) * (q1 - 1.0 / r2));
        return exp((an + 2) * log_series(rm1)) / pp1 + oscillatory(r2, p2, 3, n);
    }
    return pow(r1, (double)(an + 2)) / pp6(r1, c) + oscillatory(r2, p2, 3, n);
}

// ---------------------------------------------------------------- LGF8 (9-point stencil)
__device__ inline void lgf8_roots(double c, zc r[3]) {
    const double tmp1 = 1968941520. + c * (-879221700. + c * (223915104. - c * 44089920));
    const zc xi = zpow(1520225. - 273420. * c + 35. * zsqrt(Z(tmp1)), 1. / 3.);
    const double del = (xi + (-4655. + 3780. * c) / xi).x;
    const zc eta = zsqrt(Z(del / 9. - 434. / 81.));
    const zc s1 = zsqrt(-868. / 81. + 81088. / (729. * eta) - del / 9.);
    const zc s3 = zsqrt(-868. / 81. - 81088. / (729. * eta) - del / 9.);
    const zc lam[3] = {0.5 * (32. / 9. + eta - s1), 0.5 * (32. / 9. + eta + s1), 0.5 * (32. / 9. - eta - s3)};
    for (int i = 0; i < 3; ++i) r[i] = lam[i] - zsqrt(lam[i] + 1.0) * zsqrt(lam[i] - 1.0);
}

__device__ inline double lgf8(int n, double c) {
    const int an = abs(n);
    const double cstar = 3.204471924659902;
    if (c == 0.0) {
        const double rho1 = 1.2185576475724652e-01, th1 = 1.4667413886166037e+00, a1 = 8.2123351081853858e-02;
        const double phi1 = -6.5666289805823130e-01, r2 = 9.6191214171019512e-02, a2 = 4.0692417408429382e-02;
        return -0.5 * an + a1 * pow(rho1, (double)an) * sin(an * th1 + phi1) - a1 * sin(phi1) + a2 * (1.0 - pow(r2, (double)an));
    }
    if (c >= cstar - 1e-5 && c < cstar + 1e-5) {
        const double a0[2] = {-0.1932304295173025, -9.940958723693284e-2};
        const double a1[4] = {5.528645180523051e-2, 6.381749748906844e-2, 1.920895723993029e-2, 1.647044339102893e-3};
        const double a2[6] = {-1.246195963786745e-2, -2.200316066032414e-2, -1.156690496243602e-2, -2.513956535483380e-3,
                              -2.386943138091703e-4, -8.186599895557273e-6};
        const double a3[8] = {2.586595339831205e-3, 5.946351585490818e-3, 4.392324394119772e-3, 1.460419122054276e-3,
                              2.498408821419240e-4, 2.281049273902400e-5, 1.054600142736557e-6, 1.937682182122062e-8};
        const double a4[10] = {-6.143387386724980e-4, -1.461770070530813e-3, -1.338631620906462e-3, -5.893614275050890e-4,
                               -1.419718637870522e-4, -2.006233681173800e-5, -1.705558618042543e-6, -8.568226736629197e-8,
                               -2.340119751996688e-9, -2.675335915571021e-11};
        const double u0[1] = {0.0015031218476240784};
        const double u1[2] = {-0.013198947960911374, -0.00309497626043345};
        const double u2[3] = {0.002223792419320104, 0.0003211726758356002, -3.489943855291188e-6};
        const double u3[4] = {8.218756082933073e-5, 0.00012939734109457704, 2.076196709989474e-5, 7.970739601754506e-7};
        const double u4[5] = {-0.00011284539233578474, -4.455888056601662e-5, -4.596415525190604e-6, -1.2515613302441402e-7,
                              7.499072573978986e-10};
        const double v0[1] = {-0.07869060869097218};
        const double v1[2] = {0.005694070346472886, -0.00011828157312623746};
        const double v2[3] = {0.001748394270280815, 0.0007853940979982054, 6.08419435502199e-5};
        const double v3[4] = {-0.000574565978306078, -0.000152486888729598, -8.030910109571855e-6, 6.101311014540467e-8};
        const double v4[5] = {4.706634682161246e-5, -8.921284296708267e-6, -4.142946014756904e-6, -3.42884013573887e-7,
                              -7.828815619884859e-9};
        const double r0 = 1.4016094393066413e-01, rho1 = 1.2718191072648583e-01, theta1 = 1.5912866598657263e+00;
        const double r0n = pow(r0, (double)an), p1n = pow(rho1, (double)an);
        const double cn = cos(an * theta1), sn = sin(an * theta1), nr = (double)an;
        const double g[5] = {r0n * horn(a0, 2, nr) + p1n * (cn * horn(u0, 1, nr) + sn * horn(v0, 1, nr)),
                             r0n * horn(a1, 4, nr) + p1n * (cn * horn(u1, 2, nr) + sn * horn(v1, 2, nr)),
                             r0n * horn(a2, 6, nr) + p1n * (cn * horn(u2, 3, nr) + sn * horn(v2, 3, nr)),
                             r0n * horn(a3, 8, nr) + p1n * (cn * horn(u3, 4, nr) + sn * horn(v3, 4, nr)),
                             r0n * horn(a4, 10, nr) + p1n * (cn * horn(u4, 5, nr) + sn * horn(v4, 5, nr))};
        return -horn(g, 5, c - cstar);
    }
    zc r[3];
    lgf8_roots(c, r);
    if (c < 1e-3) {
        const double ser[8] = {0, 0.5, 1. / 24., 1. / 720., 1. / 40320., 577. / 3628800., 389. / 6220800., 34987. / 3048192000.};
        const double rm1 = small_root_m1(ser, c), q1 = rm1 + 1.0;
        const double q2 = r[1].x;
        const double pp2 = pp8(q2, c);
        const zc pp3 = pp8(r[2], c);
        const double pp1 = 1. / 560. * vmi_series(rm1) * (q1 - q2) * (q1 - 1 / q2) * znorm((q1 - r[2]) * (q1 - 1.0 / r[2]));
        return exp((an + 3) * log_series(rm1)) / pp1 + pow(q2, (double)(an + 3)) / pp2 + oscillatory(r[2], pp3, 4, n);
    }
    if (c < cstar - 1e-5) {
        const double q1 = r[0].x, q2 = r[1].x;
        const zc r3 = r[2];
        const zc pp3 = pp8(r3, c);
        const double f1 = 560. * pow(q1, (double)(an + 3)) / ((q1 - 1. / q1) * (q1 - 1. / q2) * znorm((q1 - r3) * (q1 - 1. / r3)));
        const double f2 = 560. * pow(q2, (double)(an + 3)) / ((q2 - 1. / q1) * (q2 - 1. / q2) * znorm((q2 - r3) * (q2 - 1. / r3)));
        return (f2 - f1) / (q2 - q1) + oscillatory(r3, pp3, 4, n);
    }
    const zc r1 = r[1], r3 = r[2], cr1 = conj(r1), cr3 = conj(r3);
    const zc pp1 = Z(0.0, 1.0) / 280. * r1.y * (r1 - 1. / r1) * (r1 - 1. / cr1) * (r1 - r3) * (r1 - 1. / r3) * (r1 - cr3) *
                   (r1 - 1. / cr3);
    const zc pp3 = pp8(r3, c);
    return oscillatory(r1, pp1, 4, n) + oscillatory(r3, pp3, 4, n);
}

// ---------------------------------------------------------------- Mehrstellen 4 and 6
// (k1, k2): the two spectral wave numbers times h, |k1| >= |k2|
__device__ inline double meh4(int n, double k1, double k2, bool full) {
    const int an = abs(n);
    if (k1 == 0 && k2 == 0) return -0.5 * an - ((full && n == 0) ? 1. / 12. : 0.0);
    const double y0 = sq(sin(k1 / 2)), y1 = sq(sin(k2 / 2));
    const double a0 = -8. / 3. * (y0 * y1 - y0 - y1) + 2.0;
    const double a1 = 2. / 3. * (y0 + y1) - 1.0;
    const double lam = -a0 / (2. * a1);
    const double r = r_from_lambda(lam);
    if (!full) {
        const double base = (r / a1) * pow(r, (double)an) / (r * r - 1.0);
        return isfinite(lam) ? base : (n == 0 ? 1.0 : 0.0) / a0;
    }
    const double b0 = 5. / 6. - 1. / 3. * (y0 + y1), b1 = 1. / 12.;
    const double pr = b1 + b0 * r + b1 * r * r;
    if (isfinite(lam)) {
        const double base = pr * pow(r, (double)an) / (a1 * (r * r - 1));
        return (n == 0) ? (r / a1) * (b0 + 2. * b1 * r) / (r * r - 1.) : base;
    }
    return (n == 0 ? 1.0 : 0.0) * (b0 / a0) + (n == 1 ? 1.0 : 0.0) * (b1 / a0);
}

__device__ inline double meh6(int n, double k1, double k2, bool full) {
    const int an = abs(n);
    if (k1 == 0 && k2 == 0) return -0.5 * an - (full ? ((an == 1 ? -1. / 240. : 0.0) + (n == 0 ? 11. / 120. : 0.0)) : 0.0);
    const double y0 = sq(sin(k1 / 2)), y1 = sq(sin(k2 / 2));
    const double a0 = -8. / 5. * y0 * y1 + 8. / 3. * (y0 + y1) + 2.0;
    const double a1 = -8. / 15. * y0 * y1 + 2. / 3. * (y0 + y1) - 1.0;
    const double lam = -a0 / (2. * a1);
    const double r = r_from_lambda(lam);
    if (!full) {
        const double base = (r / a1) * pow(r, (double)an) / (r * r - 1.0);
        return isfinite(lam) ? base : -(n == 0 ? 1.0 : 0.0) / a0;
    }
    const double b0 = -1. / 15. * (sq(y0) + sq(y1)) + 8. / 45. * y0 * y1 - 11. / 45. * (y0 + y1) + 97. / 120.;
    const double b1 = -2. / 45. * (y0 + y1) + 1. / 10.;
    const double b2 = -1. / 240.;
    const double pr = b0 * sq(r) + b1 * (r + r * r * r) + b2 * (1.0 + sq(sq(r)));
    const double base = pr * pow(r, (double)(an - 1)) / (a1 * (r * r - 1.0));
    return base + (an == 1 ? 1.0 : 0.0) * (b2 / a1) + (n == 0 ? 1.0 : 0.0) * (b1 * a1 - b2 * a0) / (a1 * a1);
}

}  // namespace lgf1
}  // namespace flb
