// Register-resident power-of-two DFT passes for the DFT directions of the
// solve (PERPER and UNBUNB plans, FFTW_plan_dim.cpp:365-451 / :670-716).
//
// A line of length L is owned by P = L / R1 threads; thread p holds
// x[p + P r] for r < R1 in registers.  Stage 1 is a radix-R1 DFT in
// registers; every later Stockham stage exchanges once through shared
// memory (one padding element per 32 keeps the 64-bit accesses of a
// half-warp on distinct banks) and ends with thread p holding X[p + P r]:
// the same distribution as the input, so the inverse transform of the fused
// pass starts from registers and the Green's multiply happens in between
// without touching shared memory.  Zero padding (UNB) is never loaded and
// truncated outputs are never stored.
//
// Column passes (y or z): a CTA owns TX consecutive x columns; lanes are
// x-fastest so every global access of a warp reads TX consecutive complex
// values of a few rows.  Row passes (x): r2c / c2r of real rows through a
// complex FFT of half length (z_j = x_2j + i x_2j+1).
#include <cuda_runtime.h>

#include "cplx.cuh"
#include "fast_dft.h"
#include "pass_desc.h"

namespace flb {

template <int R, typename C>
__device__ __forceinline__ void dftr(C* v) {
    if constexpr (R == 2) dft2(v);
    else if constexpr (R == 4) dft4(v);
    else if constexpr (R == 8) dft8(v);
    else if constexpr (R == 16) dft16(v);
    else if constexpr (R == 32) dft32(v);
}

// ROWS: the lines of a CTA are thread-index-slow (row passes: p fastest),
// else thread-index-fast (column passes: the TX columns fastest).
template <typename T, int L, int R1, bool ROWS = false>
struct RegFFT {
    using C = typename CT<T>::C;
    static constexpr int P = L / R1;
    // line stride in shared memory (complex elements): the swizzled length rounded
    // to 16, plus an offset that puts the lines met by one half-warp on distinct
    // banks: a column CTA has lanes c = 0..TX-1 on TX lines (offset 2 per line,
    // the lane's p adds 0 or 1); a row CTA has P lanes per line (offset P).
    static constexpr int SC = ((L + L / 32 + 15) / 16) * 16 + (ROWS ? (P % 16) : 2);
    __device__ static __forceinline__ int sw(int i) { return i + (i >> 5); }

    template <int Ns>
    __device__ static __forceinline__ void stages(C* v, C* sm, int p, const C* __restrict__ tw) {
        constexpr int Rs = (L / Ns < R1) ? (L / Ns) : R1;
        constexpr int NB = R1 / Rs;  // butterflies per thread
        constexpr int MR = L / Rs;
        C t[R1];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = p + P * b;
            const int k = j % Ns;
#pragma unroll
            for (int r = 0; r < Rs; ++r) {
                C x = sm[sw(j + r * MR)];
                if (r > 0) {
                    const int q = (r * k * (L / (Ns * Rs))) & (L - 1);
                    x = cmul(x, tw[q]);
                }
                t[b * Rs + r] = x;
            }
            dftr<Rs>(&t[b * Rs]);
        }
        if constexpr (Ns * Rs == L) {
#pragma unroll
            for (int b = 0; b < NB; ++b)
#pragma unroll
                for (int r = 0; r < Rs; ++r) v[b + NB * r] = t[b * Rs + r];
        } else {
            __syncthreads();
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int j = p + P * b;
                const int base = (j / Ns) * Ns * Rs + (j % Ns);
#pragma unroll
                for (int r = 0; r < Rs; ++r) sm[sw(base + r * Ns)] = t[b * Rs + r];
            }
            __syncthreads();
            stages<Ns * Rs>(v, sm, p, tw);
        }
    }

    // in place on v: forward (or inverse) unnormalised DFT of the line held as v[r] = x[p + P r]
    __device__ static __forceinline__ void fft(C* v, C* sm, int p, const C* __restrict__ tw, bool inv) {
        if (inv) {
#pragma unroll
            for (int r = 0; r < R1; ++r) v[r] = cconj(v[r]);
        }
        dftr<R1>(v);
        if constexpr (P > 1) {
            __syncthreads();
#pragma unroll
            for (int k = 0; k < R1; ++k) sm[sw(p * R1 + k)] = v[k];
            __syncthreads();
            stages<R1>(v, sm, p, tw);
        }
        if (inv) {
#pragma unroll
            for (int r = 0; r < R1; ++r) v[r] = cconj(v[r]);
        }
    }
};

__device__ __forceinline__ int fold_idx(int i, int M) { return (M > 0 && 2 * i > M) ? M - i : i; }

// asynchronous global -> shared copies of single elements (LDGSTS), so the
// folded Green's values of a fused pass arrive while the forward DFT runs
template <int B>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(gmem_src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// folded Green's values staged per column: L/2 + 1 per column, row stride
// = 4 (mod 32) elements so the multiply's reads hit distinct banks
template <int L>
struct GStage {
    static constexpr int N = L / 2 + 1;
    static constexpr int S = ((N + 31) / 32) * 32 + 4;
};

// ---------------------------------------------------------------- columns
// MODE 0: forward DFT, 1: inverse DFT, 2: forward, Green multiply, inverse
// Fused passes visit the outer index in mirror pairs (0, 1, M-1, 2, M-2, ...,
// M/2) when the Green's function is folded along it, so the folded Green slab
// read for o is read again for M-o while it is still in L2.
__device__ __forceinline__ int mirror_order(int by, int nouter, int fold) {
    if (fold != nouter || fold < 4) return by;
    if (by == 0) return 0;
    if (by == nouter - 1) return nouter / 2;
    const int m = (by + 1) >> 1;
    return (by & 1) ? m : nouter - m;
}

// resident threads per SM the register budget is sized for (2 CTAs of 256
// threads for a fused or FP64 pass, 3 otherwise): the passes are bound by
// memory, and more resident lines overlap one CTA's loads with another's
// arithmetic
#ifndef FLB_COL_THREADS_PER_SM
#define FLB_COL_THREADS_PER_SM 768
#endif
#ifndef FLB_FUSED_THREADS_PER_SM
#define FLB_FUSED_THREADS_PER_SM 512
#endif
template <typename T, int THREADS, int MODE>
struct ColOcc {
    static constexpr int per_sm = (MODE == 2 || sizeof(T) == 8) ? FLB_FUSED_THREADS_PER_SM : FLB_COL_THREADS_PER_SM;
    static constexpr int want = per_sm / (THREADS < 64 ? 64 : THREADS);
    static constexpr int blocks = want < 1 ? 1 : want;
};

template <typename T, int L, int R1, int TX, int MODE>
__global__ void __launch_bounds__(TX * (L / R1), (ColOcc<T, TX * (L / R1), MODE>::blocks)) col_dft_kernel(const ColArgs a) {
    using F = RegFFT<T, L, R1>;
    using C = typename CT<T>::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int c = threadIdx.x % TX, p = threadIdx.x / TX;
    const int x = blockIdx.x * TX + c;
    const int o = (MODE == 2) ? mirror_order(blockIdx.y, a.nouter, a.f_outer) : (int)blockIdx.y;
    const int comp = blockIdx.z;
    const bool valid = x < a.nx;
    const C* in = reinterpret_cast<const C*>(a.in) + comp * a.in_cstr + (int64_t)o * a.in_ostr + x;
    C* out = reinterpret_cast<C*>(a.out) + comp * a.out_cstr + (int64_t)o * a.out_ostr + x;
    const C* tw = reinterpret_cast<const C*>(a.tw);
    T* gs = reinterpret_cast<T*>(sm + TX * F::SC);
    if constexpr (MODE == 2) {
        // the host guarantees fold length L along the line and L * g_line < 2^31
        const T* g = reinterpret_cast<const T*>(a.green) + (int64_t)fold_idx(o, a.f_outer) * a.g_outer;
        const int gl = (int)a.g_line;
        for (int e = threadIdx.x; e < TX * GStage<L>::N; e += TX * F::P) {
            const int cc = e % TX, j = e / TX, xx = blockIdx.x * TX + cc;
            T* dst = gs + cc * GStage<L>::S + j;
            if (xx < a.nx) cp_async<sizeof(T)>(dst, g + (int64_t)fold_idx(xx, a.f_x) * a.g_x + j * gl);
            else *dst = (T)0;
        }
        cp_async_commit();
    }
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int t = p + F::P * r;
        v[r] = (valid && t < a.nin) ? in[(int64_t)t * a.in_lstr] : mkc((T)0, (T)0);
    }
    C* line = sm + c * F::SC;
    F::fft(v, line, p, tw, MODE == 1);
    if constexpr (MODE == 2) {
        cp_async_wait_all();
        __syncthreads();
        const T* gc = gs + c * GStage<L>::S;
        const T nf = (T)a.normfact;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = p + F::P * r;
            const T gv = gc[2 * k > L ? L - k : k] * nf;
            v[r] = mkc(v[r].x * gv, v[r].y * gv);
        }
        // a laundered copy of the table pointer: the compiler cannot merge the second
        // DFT's twiddle loads with the first's, so those stay out of registers
        // during the multiply
        const C* tw2 = tw;
        asm("" : "+l"(tw2));
        F::fft(v, line, p, tw2, true);
    }
    if (valid) {
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int t = p + F::P * r;
            if (t < a.nout) out[(int64_t)t * a.out_lstr] = v[r];
        }
    }
}

// ---------------------------------------------------------------- rows: r2c
template <typename T, int LH, int R1, int TR>
__global__ void __launch_bounds__(TR * (LH / R1)) row_r2c_kernel(const RowArgs a) {
    using F = RegFFT<T, LH, R1, true>;
    using C = typename CT<T>::C;
    constexpr int L = 2 * LH;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int p = threadIdx.x % F::P, rr = threadIdx.x / F::P;
    const int row = blockIdx.x * TR + rr;
    const int comp = blockIdx.y;
    const bool valid = row < a.nrows;
    const int i1 = valid ? row % a.n1 : 0, i2 = valid ? row / a.n1 : 0;
    const int64_t ib = comp * a.in_cstr + (int64_t)i1 * a.in_s1 + (int64_t)i2 * a.in_s2;
    const int64_t ob = comp * a.out_cstr + (int64_t)i1 * a.out_s1 + (int64_t)i2 * a.out_s2;
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int j = p + F::P * r;
        T re = (T)0, im = (T)0;
        if (valid && 2 * j < a.nin) {
            if (a.in_f64) {
                const double* src = reinterpret_cast<const double*>(a.in) + ib;
                if (2 * j + 1 < a.nin) {
                    const double2 d = *reinterpret_cast<const double2*>(src + 2 * j);
                    re = (T)d.x; im = (T)d.y;
                } else {
                    re = (T)src[2 * j];
                }
            } else {
                const float* src = reinterpret_cast<const float*>(a.in) + ib;
                if (2 * j + 1 < a.nin) {
                    const float2 d = *reinterpret_cast<const float2*>(src + 2 * j);
                    re = (T)d.x; im = (T)d.y;
                } else {
                    re = (T)src[2 * j];
                }
            }
        }
        v[r] = mkc(re, im);
    }
    C* line = sm + rr * F::SC;
    F::fft(v, line, p, reinterpret_cast<const C*>(a.twh), false);
    // X[k] = 1/2 (Z_k + conj Z_{LH-k}) - i/2 W_L^k (Z_k - conj Z_{LH-k}),  Z_LH = Z_0
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R1; ++r) line[F::sw(p + F::P * r)] = v[r];
    __syncthreads();
    const C* tw = reinterpret_cast<const C*>(a.tw);
    if (valid) {
        C* dst = reinterpret_cast<C*>(a.out) + ob;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = p + F::P * r;
            if (k >= a.nout) continue;
            const C zk = v[r];
            const C zm = cconj(line[F::sw((LH - k) & (LH - 1))]);
            const C e = cadd(zk, zm);
            const C d = csub(zk, zm);
            const C w = cmul(tw[k], d);             // W_L^k (Z_k - conj Z_{LH-k})
            dst[k] = mkc((T)0.5 * (e.x + w.y), (T)0.5 * (e.y - w.x));
        }
        if (p == 0 && LH < a.nout) {
            const C z0 = line[0];
            dst[LH] = mkc(z0.x - z0.y, (T)0);
        }
    }
    (void)L;
}

// ---------------------------------------------------------------- rows: c2r
template <typename T, int LH, int R1, int TR>
__global__ void __launch_bounds__(TR * (LH / R1)) row_c2r_kernel(const RowArgs a) {
    using F = RegFFT<T, LH, R1, true>;
    using C = typename CT<T>::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int p = threadIdx.x % F::P, rr = threadIdx.x / F::P;
    const int row = blockIdx.x * TR + rr;
    const int comp = blockIdx.y;
    const bool valid = row < a.nrows;
    const int i1 = valid ? row % a.n1 : 0, i2 = valid ? row / a.n1 : 0;
    const int64_t ib = comp * a.in_cstr + (int64_t)i1 * a.in_s1 + (int64_t)i2 * a.in_s2;
    const int64_t ob = comp * a.out_cstr + (int64_t)i1 * a.out_s1 + (int64_t)i2 * a.out_s2;
    C* line = sm + rr * F::SC;
    const C* src = reinterpret_cast<const C*>(a.in) + ib;
    // stage the half spectrum X[0..LH] (line positions 0..LH-1, X[LH] kept aside in registers)
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int k = p + F::P * r;
        line[F::sw(k)] = valid ? src[k] : mkc((T)0, (T)0);
    }
    const C xlh = valid ? src[LH] : mkc((T)0, (T)0);
    __syncthreads();
    // Z'_k = A_k + i B_k, A = X_k + conj X_{LH-k}, B = (X_k - conj X_{LH-k}) W_L^{-k};
    // Im X_0 and Im X_LH do not enter a real inverse transform
    const C* tw = reinterpret_cast<const C*>(a.tw);
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int k = p + F::P * r;
        C xk = line[F::sw(k)];
        C xm = (k == 0) ? xlh : line[F::sw(LH - k)];
        if (k == 0) {
            xk.y = (T)0;
            xm.y = (T)0;
        }
        xm = cconj(xm);
        const C A = cadd(xk, xm);
        const C B = cmul(csub(xk, xm), cconj(tw[k]));
        v[r] = mkc(A.x - B.y, A.y + B.x);
    }
    F::fft(v, line, p, reinterpret_cast<const C*>(a.twh), true);
    if (valid) {
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int j = p + F::P * r;
            if (2 * j >= a.nout) continue;
            if (a.out_f64) {
                double* dst = reinterpret_cast<double*>(a.out) + ob;
                if (2 * j + 1 < a.nout) *reinterpret_cast<double2*>(dst + 2 * j) = make_double2((double)v[r].x, (double)v[r].y);
                else dst[2 * j] = (double)v[r].x;
            } else {
                float* dst = reinterpret_cast<float*>(a.out) + ob;
                if (2 * j + 1 < a.nout) *reinterpret_cast<float2*>(dst + 2 * j) = make_float2((float)v[r].x, (float)v[r].y);
                else dst[2 * j] = (float)v[r].x;
            }
        }
    }
}

// ---------------------------------------------------------------- dispatch
template <typename T, int L, int R1, int TX, int MODE>
static cudaError_t launch_col_t(const ColArgs& a, int ncomp, cudaStream_t s) {
    using F = RegFFT<T, L, R1>;
    const size_t smem = (size_t)TX * F::SC * sizeof(typename CT<T>::C) + (MODE == 2 ? (size_t)TX * GStage<L>::S * sizeof(T) : 0);
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(col_dft_kernel<T, L, R1, TX, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    dim3 grid((a.nx + TX - 1) / TX, a.nouter, ncomp);
    col_dft_kernel<T, L, R1, TX, MODE><<<grid, TX * F::P, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename T, int MODE>
static cudaError_t launch_col_mode(int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    constexpr int R1 = sizeof(T) == 4 ? 32 : 16;
    constexpr int TX = sizeof(T) == 4 ? 8 : 4;  // one 64-byte segment of a row per warp access
    switch (L) {
        case 64: return launch_col_t<T, 64, R1, TX, MODE>(a, ncomp, s);
        case 128: return launch_col_t<T, 128, R1, TX, MODE>(a, ncomp, s);
        case 256: return launch_col_t<T, 256, R1, TX, MODE>(a, ncomp, s);
        case 512: return launch_col_t<T, 512, R1, TX, MODE>(a, ncomp, s);
        case 1024: return launch_col_t<T, 1024, R1, TX, MODE>(a, ncomp, s);
        case 2048: return launch_col_t<T, 2048, R1, TX / 2, MODE>(a, ncomp, s);  // keep CTAs at 256 threads
    }
    return cudaErrorInvalidValue;
}

bool fast_col_supported(int L) { return L == 64 || L == 128 || L == 256 || L == 512 || L == 1024 || L == 2048; }
bool fast_row_supported(int L) { return L == 128 || L == 256 || L == 512 || L == 1024 || L == 2048 || L == 4096; }

cudaError_t launch_fast_col(int f64, int mode, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    if (f64) {
        if (mode == 0) return launch_col_mode<double, 0>(L, a, ncomp, s);
        if (mode == 1) return launch_col_mode<double, 1>(L, a, ncomp, s);
        return launch_col_mode<double, 2>(L, a, ncomp, s);
    }
    if (mode == 0) return launch_col_mode<float, 0>(L, a, ncomp, s);
    if (mode == 1) return launch_col_mode<float, 1>(L, a, ncomp, s);
    return launch_col_mode<float, 2>(L, a, ncomp, s);
}

template <typename T, int LH, int R1, bool C2R>
static cudaError_t launch_row_t(const RowArgs& a, int ncomp, cudaStream_t s) {
    using F = RegFFT<T, LH, R1, true>;
    constexpr int TR = (F::P >= 256) ? 1 : 256 / F::P;
    const size_t smem = (size_t)TR * F::SC * sizeof(typename CT<T>::C);
    static bool attr = false;
    if (!attr) {
        cudaError_t e;
        if (C2R) e = cudaFuncSetAttribute(row_c2r_kernel<T, LH, R1, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        else e = cudaFuncSetAttribute(row_r2c_kernel<T, LH, R1, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    dim3 grid((a.nrows + TR - 1) / TR, ncomp);
    if (C2R) row_c2r_kernel<T, LH, R1, TR><<<grid, TR * F::P, smem, s>>>(a);
    else row_r2c_kernel<T, LH, R1, TR><<<grid, TR * F::P, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename T, bool C2R>
static cudaError_t launch_row_len(int L, const RowArgs& a, int ncomp, cudaStream_t s) {
    constexpr int R1 = sizeof(T) == 4 ? 32 : 16;
    switch (L) {
        case 128: return launch_row_t<T, 64, R1, C2R>(a, ncomp, s);
        case 256: return launch_row_t<T, 128, R1, C2R>(a, ncomp, s);
        case 512: return launch_row_t<T, 256, R1, C2R>(a, ncomp, s);
        case 1024: return launch_row_t<T, 512, R1, C2R>(a, ncomp, s);
        case 2048: return launch_row_t<T, 1024, R1, C2R>(a, ncomp, s);
        case 4096: return launch_row_t<T, 2048, R1, C2R>(a, ncomp, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_fast_row(int f64, int c2r, int L, const RowArgs& a, int ncomp, cudaStream_t s) {
    if (f64) return c2r ? launch_row_len<double, true>(L, a, ncomp, s) : launch_row_len<double, false>(L, a, ncomp, s);
    return c2r ? launch_row_len<float, true>(L, a, ncomp, s) : launch_row_len<float, false>(L, a, ncomp, s);
}

}  // namespace flb
