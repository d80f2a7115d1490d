// General line-transform pass: any FFTW kind the reference plans use
// (r2c, c2r, c2c, DCT/DST I-IV), any BC combination, any supported length.
//
// Each CTA owns a tile of lines.  A line is gathered into shared memory
// (zero padding and the fieldstart shift of the reference's SwitchTopo are
// applied on the fly, src/SwitchTopoX_a2a.cpp:174-247), mapped onto a complex
// FFT of length M with pre/post twiddles, transformed by a mixed-radix
// Stockham FFT in shared memory, post-processed like
// FFTW_plan_dim::postprocess_plan (src/FFTW_plan_dim.cpp:497-622) and
// scattered.  In a fused pass the Green's multiply (dothemagic) and the first
// backward transform run on the same lines before anything goes back to HBM.
//
// r2r kinds as complex FFTs (u = input, n = FFTW size, W_{2M}^q = tw[q]):
//   DCT-I   M=2(n-1): even extension, Y_k = Re C_k
//   DST-I   M=2(n+1): odd extension,  Y_k = -Im C_{k+1}
//   DCT-II  M=2n: half-sample even extension, Y_k = Re(tw[k] C_k)
//   DST-II  M=2n: half-sample odd extension, Y_k = -Im(tw[k+1] C_{k+1})
//   DCT-III M=2n: c_m = a_m u_m tw[m] (a_0=1, a_m=2), Y_k = Re C_k
//   DST-III M=2n: c_m = b_{m-1} u_{m-1} tw[m] (b_{n-1}=1, b=2), Y_k = -Im C_k
//   DCT-IV  M=2n: c_m = u_m tw[m], Y_k = Re(2 e^{-i pi/(4n)} tw[k] C_k)
//   DST-IV  M=2n: c_m = u_m tw[m], Y_k = -Im(2 e^{-i pi/(4n)} tw[k] C_k)
#include <cstdio>
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "pass_desc.h"
#include "smem_attr.cuh"
#include "spectral.cuh"

namespace flb {

template <typename T>
struct SmemLayout {
    using C = typename CT<T>::C;
    int S;        // line slots in the tile
    int nraw;     // per-slot raw elements
    int M;        // per-slot FFT buffer
    int nspec;    // per-slot spectral buffer (fused)
    __device__ C* raw(unsigned char* base, int s) const { return reinterpret_cast<C*>(base) + (size_t)s * nraw; }
    __device__ C* w0(unsigned char* base, int s) const {
        return reinterpret_cast<C*>(base) + (size_t)S * nraw + (size_t)s * M;
    }
    __device__ C* w1(unsigned char* base, int s) const {
        return reinterpret_cast<C*>(base) + (size_t)S * nraw + (size_t)S * M + (size_t)s * M;
    }
    __device__ C* spec(unsigned char* base, int s) const {
        return reinterpret_cast<C*>(base) + (size_t)S * nraw + 2 * (size_t)S * M + (size_t)s * nspec;
    }
};

template <typename C>
__device__ __forceinline__ C twl(const C* tw, int q) { return tw[q]; }

// value of the padded input line b at i (input-transform units)
template <typename C>
__device__ __forceinline__ C bval(const C* raw, int nsrc, int fieldstart, int i) {
    const int j = i - fieldstart;
    if (j >= 0 && j < nsrc) return raw[j];
    return mkc((decltype(raw[0].x))0, (decltype(raw[0].x))0);
}

// complex FFT input c[m] of one line (already conjugated for inverse DFTs)
template <typename T>
__device__ __forceinline__ typename CT<T>::C pre_value(const LineSpec& sp, const LineStage& st, const typename CT<T>::C* raw,
                                                       int nsrc, int m, const typename CT<T>::C* tw) {
    using C = typename CT<T>::C;
    const T z = (T)0;
    const int M = st.M, n = sp.n_in, fi = sp.fi, fs = st.fieldstart;
    auto u = [&](int t) { return bval(raw, nsrc, fs, fi + t); };
    switch (sp.kind) {
        case LK_R2C: return mkc(u(m).x, z);
        case LK_C2C: { C v = u(m); return sp.sign > 0 ? cconj(v) : v; }
        case LK_C2R: {
            C v = (m <= M / 2) ? u(m) : cconj(u(M - m));
            return cconj(v);
        }
        case LK_DCT1: return mkc(m < n ? u(m).x : u(M - m).x, z);
        case LK_DST1: {
            if (m == 0 || m == n + 1) return mkc(z, z);
            if (m <= n) return mkc(u(m - 1).x, z);
            return mkc(-u(M - m - 1).x, z);
        }
        case LK_DCT2: return mkc(m < n ? u(m).x : u(2 * n - 1 - m).x, z);
        case LK_DST2: return mkc(m < n ? u(m).x : -u(2 * n - 1 - m).x, z);
        case LK_DCT3: {
            if (m >= n) return mkc(z, z);
            const T a = (m == 0) ? (T)1 : (T)2;
            return cscale(twl(tw, m), a * u(m).x);
        }
        case LK_DST3: {
            if (m == 0 || m > n) return mkc(z, z);
            const T b = (m - 1 == n - 1) ? (T)1 : (T)2;
            return cscale(twl(tw, m), b * u(m - 1).x);
        }
        case LK_DCT4:
        case LK_DST4:
            if (m >= n) return mkc(z, z);
            return cscale(twl(tw, m), u(m).x);
        default: return mkc(z, z);
    }
}

// number of transform outputs written at fo
__device__ __forceinline__ int n_written(const LineSpec& sp) {
    switch (sp.kind) {
        case LK_R2C: return sp.n_in / 2 + 1;
        default: return sp.n_in;
    }
}

// output line value o[i] before post-processing (output-transform units)
template <typename T>
__device__ __forceinline__ typename CT<T>::C out_value(const LineSpec& sp, const LineStage& st, const typename CT<T>::C* Cv,
                                                       const typename CT<T>::C* raw, int nsrc, int i,
                                                       const typename CT<T>::C* tw, typename CT<T>::C ph4) {
    using C = typename CT<T>::C;
    const T z = (T)0;
    const int k = i - sp.fo;
    if (k < 0 || k >= n_written(sp)) {
        // untouched by the in-place transform: keeps the padded input (same units only)
        if (sp.kind == LK_R2C || sp.kind == LK_C2R) return mkc(z, z);
        return bval(raw, nsrc, st.fieldstart, i);
    }
    switch (sp.kind) {
        case LK_R2C: return Cv[k];
        case LK_C2C: return sp.sign > 0 ? cconj(Cv[k]) : Cv[k];
        case LK_C2R: return mkc(Cv[k].x, z);
        case LK_DCT1: return mkc(Cv[k].x, z);
        case LK_DST1: return mkc(-Cv[k + 1].y, z);
        case LK_DCT2: return mkc(cmul(twl(tw, k), Cv[k]).x, z);
        case LK_DST2: return mkc(-cmul(twl(tw, k + 1), Cv[k + 1]).y, z);
        case LK_DCT3: return mkc(Cv[k].x, z);
        case LK_DST3: return mkc(-Cv[k].y, z);
        case LK_DCT4: { C w = cmul(ph4, cmul(twl(tw, k), Cv[k])); return mkc((T)2 * w.x, z); }
        case LK_DST4: { C w = cmul(ph4, cmul(twl(tw, k), Cv[k])); return mkc(-(T)2 * w.y, z); }
        default: return mkc(z, z);
    }
}

template <typename T>
__device__ __forceinline__ typename CT<T>::C post_value(const LineSpec& sp, const LineStage& st, const typename CT<T>::C* Cv,
                                                        const typename CT<T>::C* raw, int nsrc, int i,
                                                        const typename CT<T>::C* tw, typename CT<T>::C ph4) {
    using C = typename CT<T>::C;
    const int c = sp.postpro;
    const bool first = c & PP_NULL_FIRST, last = c & PP_NULL_LAST, period = c & PP_ENFORCE_PERIOD;
    if (first && i == 0) return mkc((T)0, (T)0);
    if (last && i == st.n_o - 1) return mkc((T)0, (T)0);
    if (period && !first && !last && i == sp.nfftw) return out_value<T>(sp, st, Cv, raw, nsrc, 0, tw, ph4);
    return out_value<T>(sp, st, Cv, raw, nsrc, i, tw, ph4);
}

// ---------------------------------------------------------------- Stockham
template <typename C, int R>
__device__ __forceinline__ void bfly(C* v) {
    if constexpr (R == 2) dft2(v);
    else if constexpr (R == 3) dft3(v);
    else if constexpr (R == 4) dft4(v);
    else if constexpr (R == 5) dft5(v);
    else if constexpr (R == 8) dft8(v);
    else if constexpr (R == 16) dft16(v);
}

template <typename C, int R>
__device__ void stockham_stage(const LineStage& st, const SmemLayout<decltype(C().x)>& L, unsigned char* sm, bool from0,
                               int Ns, const C* tw) {
    const int M = st.M;
    const int MR = M / R;
    const int stride_tw = M / (Ns * R);
    const int total = L.S * MR;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        const int s = w / MR, j = w - s * MR;
        const C* src = from0 ? L.w0(sm, s) : L.w1(sm, s);
        C* dst = from0 ? L.w1(sm, s) : L.w0(sm, s);
        const int k = j % Ns;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[j + r * MR];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const int q = (r * k * stride_tw) % M;
                v[r] = cmul(v[r], tw[2 * q]);
            }
        }
        bfly<C, R>(v);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
    }
}

// any radix up to 64 by direct summation (rare lengths only)
template <typename C>
__device__ void stockham_stage_generic(const LineStage& st, const SmemLayout<decltype(C().x)>& L, unsigned char* sm, bool from0,
                                       int Ns, int R, const C* tw) {
    const int M = st.M;
    const int MR = M / R;
    const int stride_tw = M / (Ns * R);
    const int total = L.S * MR;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        const int s = w / MR, j = w - s * MR;
        const C* src = from0 ? L.w0(sm, s) : L.w1(sm, s);
        C* dst = from0 ? L.w1(sm, s) : L.w0(sm, s);
        const int k = j % Ns;
        C v[64];
        for (int r = 0; r < R; ++r) {
            v[r] = src[j + r * MR];
            if (Ns > 1 && r > 0) v[r] = cmul(v[r], tw[2 * ((r * k * stride_tw) % M)]);
        }
        const int base = (j / Ns) * Ns * R + k;
        for (int q = 0; q < R; ++q) {
            C acc = v[0];
            for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(v[r], tw[2 * (((r * q) % R) * MR)]));
            dst[base + q * Ns] = acc;
        }
    }
}

// runs all stages; returns true when the result is in w0
template <typename T>
__device__ bool fft_all(const LineStage& st, const SmemLayout<T>& L, unsigned char* sm) {
    using C = typename CT<T>::C;
    const C* tw = reinterpret_cast<const C*>(st.tw);
    bool from0 = true;
    int Ns = 1;
    for (int s = 0; s < st.nrad; ++s) {
        const int R = st.radix[s];
        switch (R) {
            case 2: stockham_stage<C, 2>(st, L, sm, from0, Ns, tw); break;
            case 3: stockham_stage<C, 3>(st, L, sm, from0, Ns, tw); break;
            case 4: stockham_stage<C, 4>(st, L, sm, from0, Ns, tw); break;
            case 5: stockham_stage<C, 5>(st, L, sm, from0, Ns, tw); break;
            case 8: stockham_stage<C, 8>(st, L, sm, from0, Ns, tw); break;
            case 16: stockham_stage<C, 16>(st, L, sm, from0, Ns, tw); break;
            default: stockham_stage_generic<C>(st, L, sm, from0, Ns, R, tw); break;
        }
        __syncthreads();
        from0 = !from0;
        Ns *= R;
    }
    return from0;
}

// ---------------------------------------------------------------- helpers
struct SlotPos {
    int comp, ia, ib;
};

__device__ __forceinline__ void axes_of(int axis, int& a, int& b) {
    a = (axis == 0) ? 1 : 0;
    b = (axis == 2) ? 1 : 2;
}

template <typename T>
__device__ __forceinline__ T load_elem(const void* p, int64_t off, int f64, int cplx, int part) {
    if (f64) return (T)(reinterpret_cast<const double*>(p)[cplx ? 2 * off + part : off]);
    return (T)(reinterpret_cast<const float*>(p)[cplx ? 2 * off + part : off]);
}

// ---------------------------------------------------------------- kernel
template <typename T>
__global__ void __launch_bounds__(256) line_pass_kernel(const PassArgs A, int in_f64, int out_f64) {
    using C = typename CT<T>::C;
    extern __shared__ __align__(16) unsigned char sm[];
    const int fused = A.fused;
    const LineStage& S0 = A.st[0];
    const int ncg = A.comps_together ? A.ncomp : 1;   // components per position inside the CTA
    const int TL = A.lines_per_cta;                   // positions (or slots) per CTA
    const int S = TL * ncg;                           // slots
    const int Mmax = fused ? max(S0.M, A.st[1].M) : S0.M;
    SmemLayout<T> L{S, A.n_src, Mmax, fused ? S0.n_o : 0};
    int ax_a, ax_b;
    axes_of(A.axis, ax_a, ax_b);
    const int64_t total_slots = A.comps_together ? (int64_t)A.nlines * ncg : (int64_t)A.nlines * A.ncomp;
    const int64_t slot0 = (int64_t)blockIdx.x * S;

    auto slot_pos = [&](int s, bool& valid) {
        SlotPos p;
        int64_t g;
        if (A.comps_together) {
            const int c = s / TL, l = s - c * TL;
            const int64_t pos = (int64_t)blockIdx.x * TL + l;
            valid = pos < A.nlines;
            p.comp = c;
            g = pos;
        } else {
            g = slot0 + s;
            valid = g < total_slots;
            p.comp = (int)(g / A.nlines);
            g -= (int64_t)p.comp * A.nlines;
        }
        p.ia = (int)(g % A.n_a);
        p.ib = (int)(g / A.n_a);
        return p;
    };

    // ---- 1. gather source lines
    {
        const int n = A.n_src;
        const bool along = (A.in_str[A.axis] == 1);
        const int total = S * n;
        for (int w = threadIdx.x; w < total; w += blockDim.x) {
            int s, t;
            if (along) { s = w / n; t = w - s * n; } else { t = w / S; s = w - t * S; }
            bool valid;
            SlotPos p = slot_pos(s, valid);
            C v = mkc((T)0, (T)0);
            if (valid) {
                const int64_t off = p.comp * A.in_cstr + (int64_t)p.ia * A.in_str[ax_a] + (int64_t)p.ib * A.in_str[ax_b] +
                                    (int64_t)t * A.in_str[A.axis];
                const int cp = S0.in_cplx;
                v.x = load_elem<T>(A.in, off, in_f64, cp, 0);
                if (cp) v.y = load_elem<T>(A.in, off, in_f64, cp, 1);
            }
            L.raw(sm, s)[t] = v;
        }
    }
    __syncthreads();

    for (int stage = 0; stage <= fused; ++stage) {
        const LineStage& ST = A.st[stage];
        const C* tw = reinterpret_cast<const C*>(ST.tw);
        const int nsrc = stage == 0 ? A.n_src : S0.n_o;
        // ---- 2. pre: build the complex FFT input
        {
            const int M = ST.M;
            const int total = S * M;
            for (int w = threadIdx.x; w < total; w += blockDim.x) {
                const int s = w / M, m = w - s * M;
                bool valid;
                SlotPos p = slot_pos(s, valid);
                const LineSpec& sp = ST.spec[p.comp % A.lda];
                const C* src = stage == 0 ? L.raw(sm, s) : L.spec(sm, s);
                L.w0(sm, s)[m] = pre_value<T>(sp, ST, src, nsrc, m, tw);
            }
        }
        __syncthreads();
        // ---- 3. FFT
        const bool in0 = fft_all<T>(ST, L, sm);
        // ---- 4. post: output line (to the spectral buffer, or scattered)
        if (stage == 0 && fused) {
            const int n = ST.n_o;
            const int total = S * n;
            for (int w = threadIdx.x; w < total; w += blockDim.x) {
                const int s = w / n, i = w - s * n;
                bool valid;
                SlotPos p = slot_pos(s, valid);
                const LineSpec& sp = ST.spec[p.comp % A.lda];
                const C* Cv = in0 ? L.w0(sm, s) : L.w1(sm, s);
                const C ph4 = mkc((T)0, (T)0);
                C ph = ph4;
                if (sp.kind == LK_DCT4 || sp.kind == LK_DST4) {
                    const double a = -3.14159265358979323846 / (4.0 * sp.n_in);
                    ph = mkc((T)cos(a), (T)sin(a));
                }
                L.spec(sm, s)[i] = post_value<T>(sp, ST, Cv, L.raw(sm, s), nsrc, i, tw, ph);
            }
            __syncthreads();
            // ---- 5. spectral multiply
            const MultSpec& G = A.mult;
            const T* green = reinterpret_cast<const T*>(G.green);
            if (G.mode == 1) {
                for (int w = threadIdx.x; w < total; w += blockDim.x) {
                    const int s = w / n, i = w - s * n;
                    bool valid;
                    SlotPos p = slot_pos(s, valid);
                    if (!valid) continue;
                    int idx[3];
                    idx[A.axis] = i; idx[ax_a] = p.ia; idx[ax_b] = p.ib;
                    int64_t go = 0;
                    for (int d = 0; d < 3; ++d) go += (int64_t)gfold(idx[d], G.gfold[d]) * G.gstr[d];
                    const T g = green[go] * (T)G.normfact;
                    C v = L.spec(sm, s)[i];
                    L.spec(sm, s)[i] = mkc(v.x * g, v.y * g);
                }
            } else if (G.mode == 2) {
                // three components of one position live in slots c*TL + l
                const int totalp = TL * n;
                for (int w = threadIdx.x; w < totalp; w += blockDim.x) {
                    const int l = w / n, i = w - l * n;
                    bool valid;
                    SlotPos p = slot_pos(l, valid);
                    if (!valid) continue;
                    int idx[3];
                    idx[A.axis] = i; idx[ax_a] = p.ia; idx[ax_b] = p.ib;
                    int64_t go = 0;
                    double kk[3];
                    for (int d = 0; d < 3; ++d) {
                        go += (int64_t)gfold(idx[d], G.gfold[d]) * G.gstr[d];
                        kk[d] = (double)symid(idx[d], G.symstart[d]) + G.koffset[d];
                    }
                    const double g = (double)green[go] * G.normfact;
                    // kc(d, c) = symbol of (is_d + koffset_d) * kfact[d][c] (complex)
                    auto kc = [&](int d, int c) {
                        return make_double2(fd_symbol(G.odiff, kk[d] * G.kfact[d][c][0], G.hgrid[d]),
                                            fd_symbol(G.odiff, kk[d] * G.kfact[d][c][1], G.hgrid[d]));
                    };
                    C* f0p = L.spec(sm, 0 * TL + l);
                    C* f1p = L.spec(sm, 1 * TL + l);
                    C* f2p = L.spec(sm, 2 * TL + l);
                    const double2 f0 = make_double2(f0p[i].x, f0p[i].y);
                    const double2 f1 = make_double2(f1p[i].x, f1p[i].y);
                    const double2 f2 = make_double2(f2p[i].x, f2p[i].y);
                    const double2 r0 = csub(cmul(f2, kc(1, 2)), cmul(f1, kc(2, 1)));
                    const double2 r1 = csub(cmul(f0, kc(2, 0)), cmul(f2, kc(0, 2)));
                    const double2 r2 = csub(cmul(f1, kc(0, 1)), cmul(f0, kc(1, 0)));
                    f0p[i] = mkc((T)(r0.x * g), (T)(r0.y * g));
                    f1p[i] = mkc((T)(r1.x * g), (T)(r1.y * g));
                    f2p[i] = mkc((T)(r2.x * g), (T)(r2.y * g));
                }
            }
            __syncthreads();
            continue;
        }
        // ---- scatter the kept part of the output line
        {
            const int n = ST.n_store;
            const bool along = (A.out_str[A.axis] == 1);
            const int total = S * n;
            for (int w = threadIdx.x; w < total; w += blockDim.x) {
                int s, t;
                if (along) { s = w / n; t = w - s * n; } else { t = w / S; s = w - t * S; }
                bool valid;
                SlotPos p = slot_pos(s, valid);
                if (!valid) continue;
                const LineSpec& sp = ST.spec[p.comp % A.lda];
                const C* Cv = in0 ? L.w0(sm, s) : L.w1(sm, s);
                C ph = mkc((T)0, (T)0);
                if (sp.kind == LK_DCT4 || sp.kind == LK_DST4) {
                    const double a = -3.14159265358979323846 / (4.0 * sp.n_in);
                    ph = mkc((T)cos(a), (T)sin(a));
                }
                const C* src = stage == 0 ? L.raw(sm, s) : L.spec(sm, s);
                const C v = post_value<T>(sp, ST, Cv, src, nsrc, ST.store_off + t, tw, ph);
                const int64_t off = p.comp * A.out_cstr + (int64_t)p.ia * A.out_str[ax_a] + (int64_t)p.ib * A.out_str[ax_b] +
                                    (int64_t)t * A.out_str[A.axis];
                if (out_f64) {
                    double* o = reinterpret_cast<double*>(A.out);
                    if (ST.out_cplx) { o[2 * off] = (double)v.x; o[2 * off + 1] = (double)v.y; }
                    else o[off] = (double)v.x;
                } else {
                    float* o = reinterpret_cast<float*>(A.out);
                    if (ST.out_cplx) { o[2 * off] = (float)v.x; o[2 * off + 1] = (float)v.y; }
                    else o[off] = (float)v.x;
                }
            }
        }
    }
}

// ---------------------------------------------------------------- host side
size_t line_pass_smem(const PassArgs& A, int elem_bytes) {
    const int ncg = A.comps_together ? A.ncomp : 1;
    const int S = A.lines_per_cta * ncg;
    const int Mmax = A.fused ? (A.st[0].M > A.st[1].M ? A.st[0].M : A.st[1].M) : A.st[0].M;
    const size_t cbytes = 2 * (size_t)elem_bytes;
    return (size_t)S * ((size_t)A.n_src + 2 * (size_t)Mmax + (A.fused ? (size_t)A.st[0].n_o : 0)) * cbytes;
}

template <typename T>
cudaError_t launch_line_pass_t(const PassArgs& A, int in_f64, int out_f64, cudaStream_t stream) {
    const size_t smem = line_pass_smem(A, sizeof(T));
    static std::atomic<unsigned long long> attr{0};
    if (cudaError_t e = smem_attr_once(attr, line_pass_kernel<T>, 227 * 1024); e != cudaSuccess) return e;
    const int ncg = A.comps_together ? A.ncomp : 1;
    int64_t nblocks;
    if (A.comps_together) nblocks = ((int64_t)A.nlines + A.lines_per_cta - 1) / A.lines_per_cta;
    else nblocks = ((int64_t)A.nlines * A.ncomp + A.lines_per_cta - 1) / A.lines_per_cta;
    (void)ncg;
    if (nblocks <= 0) return cudaSuccess;
    line_pass_kernel<T><<<(unsigned)nblocks, 256, smem, stream>>>(A, in_f64, out_f64);
    return cudaGetLastError();
}

cudaError_t launch_line_pass(const PassArgs& A, int compute_f64, int in_f64, int out_f64, cudaStream_t stream) {
    if (compute_f64) return launch_line_pass_t<double>(A, in_f64, out_f64, stream);
    return launch_line_pass_t<float>(A, in_f64, out_f64, stream);
}

}  // namespace flb
