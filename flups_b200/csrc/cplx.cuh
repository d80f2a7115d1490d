// Small complex helpers and fixed-radix DFT butterflies (forward sign,
// W_R = exp(-2 pi i / R)); inverse transforms conjugate on the way in and out.
#pragma once
#include <cuda_runtime.h>

namespace flb {

template <typename T> struct CT;
template <> struct CT<float> { using C = float2; };
template <> struct CT<double> { using C = double2; };

__device__ __forceinline__ float2 mkc(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 mkc(double x, double y) { return make_double2(x, y); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mkc(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mkc(a.x - b.x, a.y - b.y); }
#ifndef FLB_PAIRED_FP32
#define FLB_PAIRED_FP32 1
#endif
#if FLB_PAIRED_FP32 && defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
// FP32 complex additions as one paired instruction (per component the same
// rounding as the scalar operation); a - b as b * (-1) + a, exact in the product
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
#endif
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mkc(a.x, -a.y); }
// a * (-i)
template <typename C> __device__ __forceinline__ C cmul_mi(C a) { return mkc(a.y, -a.x); }
template <typename C, typename S> __device__ __forceinline__ C cscale(C a, S s) { return mkc(a.x * s, a.y * s); }

template <bool INV = false, typename C> __device__ __forceinline__ void dft2(C* v) {
    C t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
}

// t -/+ i d, component by component (no swapped pair is formed)
template <typename C> __device__ __forceinline__ C csub_i(C t, C d) { return mkc(t.x + d.y, t.y - d.x); }
template <typename C> __device__ __forceinline__ C cadd_i(C t, C d) { return mkc(t.x - d.y, t.y + d.x); }

// a * conj(w)
template <typename C> __device__ __forceinline__ C cmulc(C a, C w) {
    return mkc(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}
// a * (+i)
template <typename C> __device__ __forceinline__ C cmul_pi(C a) { return mkc(-a.y, a.x); }

// INV: the inverse butterfly (conjugate roots of unity), written out so that
// an inverse transform needs no conjugation of its input and output
template <bool INV = false, typename C> __device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
    const C t0 = cadd(a0, a2), t1 = csub(a0, a2);
    const C t2 = cadd(a1, a3), d = csub(a1, a3);
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    if constexpr (INV) {
        a1 = cadd_i(t1, d);  // t1 + i d
        a3 = csub_i(t1, d);
    } else {
        a1 = csub_i(t1, d);  // t1 + (-i) d
        a3 = cadd_i(t1, d);
    }
}
template <bool INV = false, typename C> __device__ __forceinline__ void dft4(C* v) { dft4<INV>(v[0], v[1], v[2], v[3]); }

// sqrt(1/2), cos(pi/8), sin(pi/8)
#define FLB_R2 0.70710678118654752440
#define FLB_C8 0.92387953251128675613
#define FLB_S8 0.38268343236508977173

template <bool INV = false, typename C> __device__ __forceinline__ void dft8(C* v) {
    using S = decltype(v[0].x);
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    const S r2 = (S)FLB_R2;
    if constexpr (INV) {
        o1 = mkc((o1.x - o1.y) * r2, (o1.x + o1.y) * r2);   // * conj(W8^1)
        o3 = mkc(-(o3.x + o3.y) * r2, (o3.x - o3.y) * r2);  // * conj(W8^3)
    } else {
        o1 = mkc((o1.x + o1.y) * r2, (o1.y - o1.x) * r2);   // * W8^1
        o3 = mkc((o3.y - o3.x) * r2, -(o3.x + o3.y) * r2);  // * W8^3
    }
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    if constexpr (INV) {
        v[2] = cadd_i(e2, o2); v[6] = csub_i(e2, o2);    // o2 * conj(W8^2) = i o2
    } else {
        v[2] = csub_i(e2, o2); v[6] = cadd_i(e2, o2);    // o2 * W8^2 = -i o2
    }
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

// W16^m = (cos(pi m/8), -sin(pi m/8)), m in 0..9
template <typename S> __device__ __forceinline__ void w16(int m, S& c, S& s) {
    switch (m) {
        case 0: c = (S)1; s = (S)0; break;
        case 1: c = (S)FLB_C8; s = -(S)FLB_S8; break;
        case 2: c = (S)FLB_R2; s = -(S)FLB_R2; break;
        case 3: c = (S)FLB_S8; s = -(S)FLB_C8; break;
        case 4: c = (S)0; s = (S)-1; break;
        case 6: c = -(S)FLB_R2; s = -(S)FLB_R2; break;
        case 9: c = -(S)FLB_C8; s = (S)FLB_S8; break;
        default: c = (S)0; s = (S)0; break;
    }
}

template <bool INV = false, typename C> __device__ __forceinline__ void dft16(C* v) {
    using S = decltype(v[0].x);
    // inner DFT4 over j1 of a[j2 + 4 j1], twiddle W16^{j2 k1}, outer DFT4 over j2
#pragma unroll
    for (int j2 = 0; j2 < 4; ++j2) dft4<INV>(v[j2], v[j2 + 4], v[j2 + 8], v[j2 + 12]);
#pragma unroll
    for (int j2 = 1; j2 < 4; ++j2) {
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) {
            if (j2 * k1 == 4) {
                v[j2 + 4 * k1] = INV ? cmul_pi(v[j2 + 4 * k1]) : cmul_mi(v[j2 + 4 * k1]);
            } else {
                S c, s;
                w16<S>(j2 * k1, c, s);
                v[j2 + 4 * k1] = cmul(v[j2 + 4 * k1], mkc(c, INV ? -s : s));
            }
        }
    }
    C t[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        C a0 = v[0 + 4 * k1], a1 = v[1 + 4 * k1], a2 = v[2 + 4 * k1], a3 = v[3 + 4 * k1];
        dft4<INV>(a0, a1, a2, a3);
        t[k1 + 0] = a0; t[k1 + 4] = a1; t[k1 + 8] = a2; t[k1 + 12] = a3;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = t[i];
}

// W32^m = (cos(pi m/16), -sin(pi m/16)) for the m = n1*k2 products of dft32
template <typename S> __device__ __forceinline__ void w32(int m, S& c, S& s) {
    switch (m) {
        case 0: c = (S)1; s = (S)0; break;
        case 1: c = (S)0.98078528040323044913; s = -(S)0.19509032201612826785; break;
        case 2: c = (S)0.92387953251128675613; s = -(S)0.38268343236508977173; break;
        case 3: c = (S)0.83146961230254523708; s = -(S)0.55557023301960222474; break;
        case 4: c = (S)0.70710678118654752440; s = -(S)0.70710678118654752440; break;
        case 5: c = (S)0.55557023301960222474; s = -(S)0.83146961230254523708; break;
        case 6: c = (S)0.38268343236508977173; s = -(S)0.92387953251128675613; break;
        case 7: c = (S)0.19509032201612826785; s = -(S)0.98078528040323044913; break;
        case 8: c = (S)0; s = (S)-1; break;
        case 9: c = -(S)0.19509032201612826785; s = -(S)0.98078528040323044913; break;
        case 10: c = -(S)0.38268343236508977173; s = -(S)0.92387953251128675613; break;
        case 12: c = -(S)0.70710678118654752440; s = -(S)0.70710678118654752440; break;
        case 14: c = -(S)0.92387953251128675613; s = -(S)0.38268343236508977173; break;
        case 15: c = -(S)0.98078528040323044913; s = -(S)0.19509032201612826785; break;
        case 18: c = -(S)0.92387953251128675613; s = (S)0.38268343236508977173; break;
        case 21: c = -(S)0.55557023301960222474; s = (S)0.83146961230254523708; break;
        default: c = (S)0; s = (S)0; break;
    }
}

// DFT32 as 4 x 8: inner DFT8 over n2 of a[n1 + 4 n2], twiddle W32^{n1 k2}, outer DFT4 over n1
template <bool INV = false, typename C> __device__ __forceinline__ void dft32(C* v) {
    using S = decltype(v[0].x);
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) {
        C a[8];
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) a[n2] = v[n1 + 4 * n2];
        dft8<INV>(a);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) v[n1 + 4 * k2] = a[k2];
    }
#pragma unroll
    for (int n1 = 1; n1 < 4; ++n1) {
#pragma unroll
        for (int k2 = 1; k2 < 8; ++k2) {
            if (n1 * k2 == 8) {
                v[n1 + 4 * k2] = INV ? cmul_pi(v[n1 + 4 * k2]) : cmul_mi(v[n1 + 4 * k2]);
            } else {
                S c, s;
                w32<S>(n1 * k2, c, s);
                v[n1 + 4 * k2] = cmul(v[n1 + 4 * k2], mkc(c, INV ? -s : s));
            }
        }
    }
    C t[32];
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) {
        C a0 = v[0 + 4 * k2], a1 = v[1 + 4 * k2], a2 = v[2 + 4 * k2], a3 = v[3 + 4 * k2];
        dft4<INV>(a0, a1, a2, a3);
        t[k2 + 0] = a0; t[k2 + 8] = a1; t[k2 + 16] = a2; t[k2 + 24] = a3;
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = t[i];
}

// Pruned butterflies for inputs whose upper half is zero (a zero-padded
// line): the additions with the zero half are skipped.
template <typename C> __device__ __forceinline__ void dft2z(C* v) { v[1] = v[0]; }

// dft4 with a2 = a3 = 0
template <typename C> __device__ __forceinline__ void dft4z(C& a0, C& a1, C& a2, C& a3) {
    const C t = a0, u = a1;
    a0 = cadd(t, u);
    a2 = csub(t, u);
    a1 = csub_i(t, u);
    a3 = cadd_i(t, u);
}
template <typename C> __device__ __forceinline__ void dft4z(C* v) { dft4z(v[0], v[1], v[2], v[3]); }

template <typename C> __device__ __forceinline__ void dft8z(C* v) {
    using S = decltype(v[0].x);
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4z(e0, e1, e2, e3);
    dft4z(o0, o1, o2, o3);
    const S r2 = (S)FLB_R2;
    o1 = mkc((o1.x + o1.y) * r2, (o1.y - o1.x) * r2);
    o3 = mkc((o3.y - o3.x) * r2, -(o3.x + o3.y) * r2);
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    v[2] = csub_i(e2, o2); v[6] = cadd_i(e2, o2);
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

template <typename C> __device__ __forceinline__ void dft16z(C* v) {
    using S = decltype(v[0].x);
#pragma unroll
    for (int j2 = 0; j2 < 4; ++j2) dft4z(v[j2], v[j2 + 4], v[j2 + 8], v[j2 + 12]);
#pragma unroll
    for (int j2 = 1; j2 < 4; ++j2) {
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) {
            if (j2 * k1 == 4) {
                v[j2 + 4 * k1] = cmul_mi(v[j2 + 4 * k1]);
            } else {
                S c, s;
                w16<S>(j2 * k1, c, s);
                v[j2 + 4 * k1] = cmul(v[j2 + 4 * k1], mkc(c, s));
            }
        }
    }
    C t[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        C a0 = v[0 + 4 * k1], a1 = v[1 + 4 * k1], a2 = v[2 + 4 * k1], a3 = v[3 + 4 * k1];
        dft4(a0, a1, a2, a3);
        t[k1 + 0] = a0; t[k1 + 4] = a1; t[k1 + 8] = a2; t[k1 + 12] = a3;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = t[i];
}

template <typename C> __device__ __forceinline__ void dft32z(C* v) {
    using S = decltype(v[0].x);
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) {
        C a[8];
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) a[n2] = v[n1 + 4 * n2];
        dft8z(a);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) v[n1 + 4 * k2] = a[k2];
    }
#pragma unroll
    for (int n1 = 1; n1 < 4; ++n1) {
#pragma unroll
        for (int k2 = 1; k2 < 8; ++k2) {
            if (n1 * k2 == 8) {
                v[n1 + 4 * k2] = cmul_mi(v[n1 + 4 * k2]);
            } else {
                S c, s;
                w32<S>(n1 * k2, c, s);
                v[n1 + 4 * k2] = cmul(v[n1 + 4 * k2], mkc(c, s));
            }
        }
    }
    C t[32];
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) {
        C a0 = v[0 + 4 * k2], a1 = v[1 + 4 * k2], a2 = v[2 + 4 * k2], a3 = v[3 + 4 * k2];
        dft4(a0, a1, a2, a3);
        t[k2 + 0] = a0; t[k2 + 8] = a1; t[k2 + 16] = a2; t[k2 + 24] = a3;
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = t[i];
}

template <bool INV = false, typename C> __device__ __forceinline__ void dft3(C* v) {
    using S = decltype(v[0].x);
    const S h = (S)0.5, s3 = (S)0.86602540378443864676;
    C a = cadd(v[1], v[2]);
    C d = INV ? cmul_pi(csub(v[1], v[2])) : cmul_mi(csub(v[1], v[2]));
    C t = csub(v[0], cscale(a, h));
    v[0] = cadd(v[0], a);
    C u = cscale(d, s3);
    v[1] = cadd(t, u);
    v[2] = csub(t, u);
}
template <bool INV = false, typename C> __device__ __forceinline__ void dft3(C& a0, C& a1, C& a2) {
    C v[3] = {a0, a1, a2};
    dft3<INV>(v);
    a0 = v[0];
    a1 = v[1];
    a2 = v[2];
}

// W24^m = (cos(pi m/12), -sin(pi m/12)) for the m = n1*k2 products of dft24
template <typename S> __device__ __forceinline__ void w24(int m, S& c, S& s) {
    switch (m) {
        case 1: c = (S)0.9659258262890682867497; s = -(S)0.2588190451025207623489; break;
        case 2: c = (S)0.8660254037844386467637; s = -(S)0.5; break;
        case 3: c = (S)0.7071067811865475244008; s = -(S)0.7071067811865475244008; break;
        case 4: c = (S)0.5; s = -(S)0.8660254037844386467637; break;
        case 5: c = (S)0.2588190451025207623489; s = -(S)0.9659258262890682867497; break;
        case 7: c = -(S)0.2588190451025207623489; s = -(S)0.9659258262890682867497; break;
        case 8: c = -(S)0.5; s = -(S)0.8660254037844386467637; break;
        case 9: c = -(S)0.7071067811865475244008; s = -(S)0.7071067811865475244008; break;
        case 10: c = -(S)0.8660254037844386467637; s = -(S)0.5; break;
        case 11: c = -(S)0.9659258262890682867497; s = -(S)0.2588190451025207623489; break;
        case 12: c = (S)-1; s = (S)0; break;
        case 13: c = -(S)0.9659258262890682867497; s = (S)0.2588190451025207623489; break;
        case 14: c = -(S)0.8660254037844386467637; s = (S)0.5; break;
        default: c = (S)1; s = (S)0; break;
    }
}

// DFT24 as 3 x 8: inner DFT8 over n2 of a[n1 + 3 n2], twiddle W24^{n1 k2},
// outer DFT3 over n1; output k2 + 8 k1.  Z: inputs 12..23 are zero (then the
// inner DFT8s see a zero upper half).
template <bool INV = false, bool Z = false, typename C> __device__ __forceinline__ void dft24(C* v) {
    using S = decltype(v[0].x);
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1) {
        C a[8];
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) a[n2] = v[n1 + 3 * n2];
        if constexpr (Z) dft8z(a);
        else dft8<INV>(a);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) v[n1 + 3 * k2] = a[k2];
    }
#pragma unroll
    for (int n1 = 1; n1 < 3; ++n1) {
#pragma unroll
        for (int k2 = 1; k2 < 8; ++k2) {
            if (n1 * k2 == 6) {
                v[n1 + 3 * k2] = INV ? cmul_pi(v[n1 + 3 * k2]) : cmul_mi(v[n1 + 3 * k2]);
            } else {
                S c, s;
                w24<S>(n1 * k2, c, s);
                v[n1 + 3 * k2] = cmul(v[n1 + 3 * k2], mkc(c, INV ? -s : s));
            }
        }
    }
    C t[24];
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) {
        C a0 = v[3 * k2], a1 = v[1 + 3 * k2], a2 = v[2 + 3 * k2];
        dft3<INV>(a0, a1, a2);
        t[k2] = a0; t[k2 + 8] = a1; t[k2 + 16] = a2;
    }
#pragma unroll
    for (int i = 0; i < 24; ++i) v[i] = t[i];
}

// W48^m = (cos(pi m/24), -sin(pi m/24)) for the m = n1*k2 products of dft48
template <typename S> __device__ __forceinline__ void w48(int m, S& c, S& s) {
    switch (m) {
        case 1: c = (S)0.9914448613738104111446; s = -(S)0.1305261922200515915484; break;
        case 2: c = (S)0.9659258262890682867497; s = -(S)0.2588190451025207623489; break;
        case 3: c = (S)0.9238795325112867561282; s = -(S)0.3826834323650897717285; break;
        case 4: c = (S)0.8660254037844386467637; s = -(S)0.5000000000000000000000; break;
        case 5: c = (S)0.7933533402912351645798; s = -(S)0.6087614290087206394161; break;
        case 6: c = (S)0.7071067811865475244008; s = -(S)0.7071067811865475244008; break;
        case 7: c = (S)0.6087614290087206394161; s = -(S)0.7933533402912351645798; break;
        case 8: c = (S)0.5000000000000000000000; s = -(S)0.8660254037844386467637; break;
        case 9: c = (S)0.3826834323650897717285; s = -(S)0.9238795325112867561282; break;
        case 10: c = (S)0.2588190451025207623489; s = -(S)0.9659258262890682867497; break;
        case 11: c = (S)0.1305261922200515915484; s = -(S)0.9914448613738104111446; break;
        case 13: c = -(S)0.1305261922200515915484; s = -(S)0.9914448613738104111446; break;
        case 14: c = -(S)0.2588190451025207623489; s = -(S)0.9659258262890682867497; break;
        case 15: c = -(S)0.3826834323650897717285; s = -(S)0.9238795325112867561282; break;
        case 16: c = -(S)0.5000000000000000000000; s = -(S)0.8660254037844386467637; break;
        case 17: c = -(S)0.6087614290087206394161; s = -(S)0.7933533402912351645798; break;
        case 18: c = -(S)0.7071067811865475244008; s = -(S)0.7071067811865475244008; break;
        case 19: c = -(S)0.7933533402912351645798; s = -(S)0.6087614290087206394161; break;
        case 20: c = -(S)0.8660254037844386467637; s = -(S)0.5000000000000000000000; break;
        case 21: c = -(S)0.9238795325112867561282; s = -(S)0.3826834323650897717285; break;
        case 22: c = -(S)0.9659258262890682867497; s = -(S)0.2588190451025207623489; break;
        case 23: c = -(S)0.9914448613738104111446; s = -(S)0.1305261922200515915484; break;
        case 24: c = (S)-1; s = (S)0; break;
        case 25: c = -(S)0.9914448613738104111446; s = (S)0.1305261922200515915484; break;
        case 26: c = -(S)0.9659258262890682867497; s = (S)0.2588190451025207623489; break;
        case 27: c = -(S)0.9238795325112867561282; s = (S)0.3826834323650897717285; break;
        case 28: c = -(S)0.8660254037844386467637; s = (S)0.5000000000000000000000; break;
        case 29: c = -(S)0.7933533402912351645798; s = (S)0.6087614290087206394161; break;
        case 30: c = -(S)0.7071067811865475244008; s = (S)0.7071067811865475244008; break;
        default: c = (S)1; s = (S)0; break;
    }
}

// DFT48 as 3 x 16: inner DFT16 over n2 of a[n1 + 3 n2], twiddle W48^{n1 k2},
// outer DFT3 over n1; output k2 + 16 k1.  Z: inputs 24..47 are zero (then the
// inner DFT16s see a zero upper half).
template <bool INV = false, bool Z = false, typename C> __device__ __forceinline__ void dft48(C* v) {
    using S = decltype(v[0].x);
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1) {
        C a[16];
#pragma unroll
        for (int n2 = 0; n2 < 16; ++n2) a[n2] = v[n1 + 3 * n2];
        if constexpr (Z) dft16z(a);
        else dft16<INV>(a);
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) v[n1 + 3 * k2] = a[k2];
    }
#pragma unroll
    for (int n1 = 1; n1 < 3; ++n1) {
#pragma unroll
        for (int k2 = 1; k2 < 16; ++k2) {
            if (n1 * k2 == 12) {
                v[n1 + 3 * k2] = INV ? cmul_pi(v[n1 + 3 * k2]) : cmul_mi(v[n1 + 3 * k2]);
            } else {
                S c, s;
                w48<S>(n1 * k2, c, s);
                v[n1 + 3 * k2] = cmul(v[n1 + 3 * k2], mkc(c, INV ? -s : s));
            }
        }
    }
    C t[48];
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) {
        C a0 = v[3 * k2], a1 = v[1 + 3 * k2], a2 = v[2 + 3 * k2];
        dft3<INV>(a0, a1, a2);
        t[k2] = a0; t[k2 + 16] = a1; t[k2 + 32] = a2;
    }
#pragma unroll
    for (int i = 0; i < 48; ++i) v[i] = t[i];
}

// W12^m = (cos(pi m/6), -sin(pi m/6))
template <typename S> __device__ __forceinline__ void w12(int m, S& c, S& s) {
    switch (m) {
        case 1: c = (S)0.8660254037844386467637; s = -(S)0.5; break;
        case 2: c = (S)0.5; s = -(S)0.8660254037844386467637; break;
        case 4: c = -(S)0.5; s = -(S)0.8660254037844386467637; break;
        case 5: c = -(S)0.8660254037844386467637; s = -(S)0.5; break;
        case 6: c = (S)-1; s = (S)0; break;
        default: c = (S)1; s = (S)0; break;
    }
}

// DFT12 as 3 x 4 (same layout as dft24); Z: inputs 6..11 are zero
template <bool INV = false, bool Z = false, typename C> __device__ __forceinline__ void dft12(C* v) {
    using S = decltype(v[0].x);
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1) {
        C a0 = v[n1], a1 = v[n1 + 3], a2 = v[n1 + 6], a3 = v[n1 + 9];
        if constexpr (Z) dft4z(a0, a1, a2, a3);
        else dft4<INV>(a0, a1, a2, a3);
        v[n1] = a0; v[n1 + 3] = a1; v[n1 + 6] = a2; v[n1 + 9] = a3;
    }
#pragma unroll
    for (int n1 = 1; n1 < 3; ++n1) {
#pragma unroll
        for (int k2 = 1; k2 < 4; ++k2) {
            if (n1 * k2 == 3) {
                v[n1 + 3 * k2] = INV ? cmul_pi(v[n1 + 3 * k2]) : cmul_mi(v[n1 + 3 * k2]);
            } else {
                S c, s;
                w12<S>(n1 * k2, c, s);
                v[n1 + 3 * k2] = cmul(v[n1 + 3 * k2], mkc(c, INV ? -s : s));
            }
        }
    }
    C t[12];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
        C a0 = v[3 * k2], a1 = v[1 + 3 * k2], a2 = v[2 + 3 * k2];
        dft3<INV>(a0, a1, a2);
        t[k2] = a0; t[k2 + 4] = a1; t[k2 + 8] = a2;
    }
#pragma unroll
    for (int i = 0; i < 12; ++i) v[i] = t[i];
}

template <typename C> __device__ __forceinline__ void dft5(C* v) {
    using S = decltype(v[0].x);
    const S c1 = (S)0.30901699437494742410, c2 = (S)-0.80901699437494742410;
    const S s1 = (S)0.95105651629515357212, s2 = (S)0.58778525229247312917;
    C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    C x0 = v[0];
    v[0] = cadd(x0, cadd(a1, a2));
    C p1 = cadd(x0, cadd(cscale(a1, c1), cscale(a2, c2)));
    C q1 = cmul_mi(cadd(cscale(b1, s1), cscale(b2, s2)));
    C p2 = cadd(x0, cadd(cscale(a1, c2), cscale(a2, c1)));
    C q2 = cmul_mi(csub(cscale(b1, s2), cscale(b2, s1)));
    v[1] = cadd(p1, q1);
    v[4] = csub(p1, q1);
    v[2] = cadd(p2, q2);
    v[3] = csub(p2, q2);
}

}  // namespace flb
