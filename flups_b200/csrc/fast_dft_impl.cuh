#pragma once
// Register-resident power-of-two DFT passes for the DFT directions of the
// solve (PERPER and UNBUNB plans, FFTW_plan_dim.cpp:365-451 / :670-716).
//
// A line of length L is owned by P = L / R1 threads; thread p holds
// x[p + P r] for r < R1 in registers.  Stage 1 is a radix-R1 DFT in
// registers; every later Stockham stage exchanges once through shared
// memory (one padding element per 32 keeps the accesses of a half-warp on
// distinct banks) and ends with thread p holding X[p + P r]: the same
// distribution as the input, so the inverse transform of the fused pass
// starts from registers and the Green's multiply happens in between without
// touching the line in shared memory.
//
// Instruction economy (the passes run close to the issue limit of the SM):
// the twiddles of a later stage come from a per-stage table laid out in the
// order the threads consume them (two per 16-byte load, no index arithmetic);
// shared-memory and global addresses are a per-thread base plus compile-time
// offsets; a line zero-padded to twice its length skips the zero half in the
// first butterflies, and outputs that are truncated are never computed.
//
// Column passes (y or z): a CTA owns TX consecutive x columns; lanes are
// x-fastest so every global access of a warp reads TX consecutive complex
// values of a few rows.  Row passes (x): r2c / c2r of real rows through a
// complex DFT of half length (z_j = x_2j + i x_2j+1).
#include <cuda_runtime.h>

#include <type_traits>

#include "cplx.cuh"
#include "fast_dft.h"
#include "pass_desc.h"
#include "smem_attr.cuh"

namespace flb {

template <int R, bool INV = false, typename C>
__device__ __forceinline__ void dftr(C* v) {
    if constexpr (R == 2) dft2<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
    else if constexpr (R == 16) dft16<INV>(v);
    else if constexpr (R == 32) dft32<INV>(v);
    else if constexpr (R == 24) dft24<INV>(v);
    else if constexpr (R == 12) dft12<INV>(v);
    else if constexpr (R == 48) dft48<INV>(v);
}

// radix-R DFT of v whose upper half is zero
template <int R, typename C>
__device__ __forceinline__ void dftz(C* v) {
    if constexpr (R == 2) dft2z(v);
    else if constexpr (R == 4) dft4z(v);
    else if constexpr (R == 8) dft8z(v);
    else if constexpr (R == 16) dft16z(v);
    else if constexpr (R == 32) dft32z(v);
    else if constexpr (R == 24) dft24<false, true>(v);
    else if constexpr (R == 12) dft12<false, true>(v);
    else if constexpr (R == 48) dft48<false, true>(v);
}

// two consecutive complex twiddles of a stage table, from shared memory
// (SM) or through the read-only data path
template <typename T, bool SM> struct TwPair;
template <bool SM> struct TwPair<float, SM> {
    __device__ static __forceinline__ void ld(const float2* p, float2& a, float2& b) {
        const float4 q = SM ? *reinterpret_cast<const float4*>(p) : __ldg(reinterpret_cast<const float4*>(p));
        a = make_float2(q.x, q.y);
        b = make_float2(q.z, q.w);
    }
};
template <bool SM> struct TwPair<double, SM> {
    __device__ static __forceinline__ void ld(const double2* p, double2& a, double2& b) {
        a = SM ? p[0] : __ldg(p);
        b = SM ? p[1] : __ldg(p + 1);
    }
};

// complex entries of the later-stage table of an n-point DFT with first radix r1
__host__ __device__ constexpr int stage_table_entries(int n, int r1) {
    int stages = 0;
    for (int Ns = r1; Ns < n; Ns *= fast_gcd(n / Ns, r1)) ++stages;
    return stages * n;
}

// ROWS: the lines of a CTA are thread-index-slow (row passes: p fastest),
// else thread-index-fast (column passes: the TX columns fastest).
// GTW: the later-stage table is read from global memory (through L1) even
// when it is small.
// WSYNC: every line lies inside one warp (ROWS with P dividing 32), so the
// exchanges synchronise the warp only
template <bool WSYNC>
__device__ __forceinline__ void line_sync() {
    if constexpr (WSYNC) __syncwarp();
    else __syncthreads();
}

template <typename T, int L, int R1, bool ROWS = false, bool GTW = false, bool WSYNC = false>
struct RegFFT {
    using C = typename CT<T>::C;
    static constexpr int P = L / R1;
    // the later-stage table is staged in shared memory when it is small
    // (FP32 lines up to 1024: one later stage, at most 8 KB)
    static constexpr int TWN = stage_table_entries(L, R1);
#ifndef FLB_TW_SMEM_MAX
#define FLB_TW_SMEM_MAX 8192
#endif
    static constexpr bool TWS = !GTW && TWN > 0 && TWN * (int)sizeof(C) <= FLB_TW_SMEM_MAX;
    static constexpr int TW_SMEM = TWS ? TWN : 0;  // complex entries of shared memory for the table
    // line stride in shared memory (complex elements): the swizzled length rounded
    // to 16, plus an offset that puts the lines met by one half-warp on distinct
    // banks: a column CTA has lanes c = 0..TX-1 on TX lines (offset 2 per line,
    // the lane's p adds 0 or 1); a row CTA has P lanes per line (offset P).
    static constexpr int SC = ((L + L / 32 + 15) / 16) * 16 + (ROWS ? (P % 16) : 2);
    __device__ static __forceinline__ int sw(int i) { return i + (i >> 5); }

    // Stockham stage with Ns-point sub-transforms done; tws = this stage's table
    template <int Ns, bool INV>
    __device__ static __forceinline__ void stages(C* v, C* sm, int p, const C* __restrict__ tws) {
        constexpr int Rs = fast_gcd(L / Ns, R1);
        static_assert(Rs >= 2 && Rs % 2 == 0, "a later stage needs an even radix");
        static_assert(!WSYNC || (ROWS && 32 % P == 0), "warp-synchronised lines lie inside one warp");
        constexpr int NB = R1 / Rs;  // butterflies per thread
        constexpr int MR = L / Rs;
        C t[R1];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = p + P * b;
            if constexpr (MR % 32 == 0) {
                // sw(j + r MR) = sw(j) + r (MR + MR/32) when MR is a multiple of 32
                const C* s0 = sm + sw(j);
#pragma unroll
                for (int r = 0; r < Rs; ++r) t[b * Rs + r] = s0[r * (MR + MR / 32)];
            } else {
#pragma unroll
                for (int r = 0; r < Rs; ++r) t[b * Rs + r] = sm[sw(j + r * MR)];
            }
            const C* tb = tws + 2 * (b * (Rs / 2) * P + p);
#pragma unroll
            for (int rp = 0; rp < Rs / 2; ++rp) {
                C w0, w1;
                TwPair<T, TWS>::ld(tb + 2 * rp * P, w0, w1);
                if constexpr (INV) {
                    if (rp > 0) t[b * Rs + 2 * rp] = cmulc(t[b * Rs + 2 * rp], w0);
                    t[b * Rs + 2 * rp + 1] = cmulc(t[b * Rs + 2 * rp + 1], w1);
                } else {
                    if (rp > 0) t[b * Rs + 2 * rp] = cmul(t[b * Rs + 2 * rp], w0);
                    t[b * Rs + 2 * rp + 1] = cmul(t[b * Rs + 2 * rp + 1], w1);
                }
            }
            dftr<Rs, INV>(&t[b * Rs]);
        }
        if constexpr (Ns * Rs == L) {
#pragma unroll
            for (int b = 0; b < NB; ++b)
#pragma unroll
                for (int r = 0; r < Rs; ++r) v[b + NB * r] = t[b * Rs + r];
        } else {
            line_sync<WSYNC>();
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const int j = p + P * b;
                const int base = (j / Ns) * Ns * Rs + (j % Ns);
                if constexpr (Ns % 32 == 0) {
                    C* d0 = sm + sw(base);
#pragma unroll
                    for (int r = 0; r < Rs; ++r) d0[r * (Ns + Ns / 32)] = t[b * Rs + r];
                } else {
#pragma unroll
                    for (int r = 0; r < Rs; ++r) sm[sw(base + r * Ns)] = t[b * Rs + r];
                }
            }
            line_sync<WSYNC>();
            stages<Ns * Rs, INV>(v, sm, p, tws + L);
        }
    }

    // in place on v: forward (INV: inverse) unnormalised DFT of the line held as
    // v[r] = x[p + P r]; ZIN: x is zero from L/2 on (v[r] = 0 for r >= R1/2);
    // Z1 (with ZIN): but for x_{L/2} = xh, held by lane 0 only, whose share of
    // lane 0's first-radix outputs is W_R1^{(R1/2) k} xh = (-1)^k xh
    template <bool ZIN, bool INV, bool Z1 = false>
    __device__ static __forceinline__ void fft(C* v, C* sm, int p, const C* __restrict__ tws, C xh = C{}) {
        static_assert(!(ZIN && INV), "zero-padded inputs are forward transforms here");
        static_assert(!Z1 || ZIN, "x_{L/2} alone is added to a zero-padded line");
        if constexpr (ZIN) dftz<R1>(v);
        else dftr<R1, INV>(v);
        if constexpr (Z1) {
            if (p == 0) {
#pragma unroll
                for (int k = 0; k < R1; ++k) v[k] = (k & 1) ? csub(v[k], xh) : cadd(v[k], xh);
            }
        }
        if constexpr (P > 1) {
            line_sync<WSYNC>();
            // sw(p R1 + k) = sw(p R1) + k for k < R1 when R1 divides 32
            if constexpr (32 % R1 == 0) {
                C* d0 = sm + sw(p * R1);
#pragma unroll
                for (int k = 0; k < R1; ++k) d0[k] = v[k];
            } else {
#pragma unroll
                for (int k = 0; k < R1; ++k) sm[sw(p * R1 + k)] = v[k];
            }
            line_sync<WSYNC>();
            stages<R1, INV>(v, sm, p, tws);
        }
    }
};

// two consecutive reals of one type as one vector
template <typename IT> struct Vec2;
template <> struct Vec2<float> { using V = float2; };
template <> struct Vec2<double> { using V = double2; };

// TMA prefetch into L2 of one box of a 4-D tensor map (a hint: no
// shared memory, no completion to wait for)
__device__ __forceinline__ void l2_prefetch_box(const CUtensorMap* m, int c0, int c1, int c2, int c3) {
    asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(reinterpret_cast<uint64_t>(m)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
}

// the input of the block `pf.dist` launches after this one (blocks launch
// in x, y, z order): columns prefetch boxes along the line (dim 1), rows
// along the row (dim 0)
template <bool ROWS>
__device__ __forceinline__ void prefetch_ahead(const Prefetch& pf, int units_per_block, int rows_n1) {
    if (pf.nbox == 0 || threadIdx.x != 0) return;
    const long long lin = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z) + pf.dist;
    const int bx = (int)(lin % gridDim.x);
    const long long rest = lin / gridDim.x;
    const int by = (int)(rest % gridDim.y), bz = (int)(rest / gridDim.y);
    if (bz >= (int)gridDim.z) return;
    if constexpr (ROWS) {
        // block bx holds rows bx * units_per_block ... ; dim 1 = i1, dim 2 = i2, dim 3 = component (grid y)
        const int row0 = bx * units_per_block;
        const int i1 = row0 % rows_n1, i2 = row0 / rows_n1;
        for (int k = 0; k < pf.nbox; ++k) l2_prefetch_box(&pf.map, k * pf.step, i1, i2, by);
    } else {
        for (int k = 0; k < pf.nbox; ++k) l2_prefetch_box(&pf.map, bx * units_per_block, k * pf.step, by, bz);
    }
}

__device__ __forceinline__ int fold_idx(int i, int M) { return (M > 0 && 2 * i > M) ? M - i : i; }

// element (line index p, outer index o) of column x in the column array of
// the rank that owns x; lstr: that array's line stride
template <typename C>
__device__ __forceinline__ C* peer_column(const ColArgs::Peers& P, int x, int o, int p, int& lstr) {
    int j = 0;
    while (j + 1 < P.n && x >= P.xs[j + 1]) ++j;
    lstr = (int)P.pitch[j];
    return reinterpret_cast<C*>(P.col[j]) + ((int64_t)(P.zs + o) * P.nl + p) * P.pitch[j] + (x - P.xs[j]);
}

// asynchronous global -> shared copies (LDGSTS): the stage twiddles and the
// folded Green's values of a fused pass arrive while the line loads are in
// flight and the first butterflies run
template <int B>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    if constexpr (B == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(gmem_src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// the stage table of F into shared memory at dst (one commit group); returns
// the table to use (dst, or the global table when F keeps it in global memory)
template <typename F>
__device__ __forceinline__ const typename F::C* stage_twiddles(const void* gtab, typename F::C* dst) {
    using C = typename F::C;
    if constexpr (F::TWS) {
        constexpr int CHUNKS = F::TWN * (int)sizeof(C) / 16;
        const char* src = reinterpret_cast<const char*>(gtab);
        char* d = reinterpret_cast<char*>(dst);
        for (int e = threadIdx.x; e < CHUNKS; e += blockDim.x) cp_async<16>(d + 16 * e, src + 16 * e);
        cp_async_commit();
        return dst;
    } else {
        return reinterpret_cast<const C*>(gtab);
    }
}

// the first n entries of a global table into shared memory at dst (no commit)
template <typename C, int n>
__device__ __forceinline__ void stage_table_part(const void* gtab, C* dst) {
    constexpr int CHUNKS = n * (int)sizeof(C) / 16;
    const char* src = reinterpret_cast<const char*>(gtab);
    char* d = reinterpret_cast<char*>(dst);
    for (int e = threadIdx.x; e < CHUNKS; e += blockDim.x) cp_async<16>(d + 16 * e, src + 16 * e);
}

// row passes keep W_L^k, k < Lh (the split of the real transform), in shared
// memory when it is small
template <typename T, int LH>
struct RowTw {
    using C = typename CT<T>::C;
    static constexpr bool SM = LH * (int)sizeof(C) <= 8192;
    static constexpr int N = SM ? LH : 0;
};

// folded Green's values of a fused CTA: line index j = 0..L/2 (the fold of
// k and L-k), TX columns x-fastest: gs[j * TX + c]
template <int L>
struct GStage {
    static constexpr int N = L / 2 + 1;
};

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

template <typename T, int L, int TX>
__device__ __forceinline__ void stage_green(const ColArgs& a, T* gs, int o) {
    constexpr int N = GStage<L>::N;
    const T* g = reinterpret_cast<const T*>(a.green) + (int64_t)fold_idx(o, a.f_outer) * a.g_outer;
    const int gl = (int)a.g_line;
    const int x0 = blockIdx.x * TX;
    constexpr int PER = 16 / (int)sizeof(T);  // values per 16-byte copy
    if constexpr (TX % PER == 0) {
        // Green rows are padded to 128 bytes and x0 is a multiple of TX, so the
        // TX values of a row are one or two aligned 16-byte pieces inside the row
        if (a.f_x == 0 && a.g_x == 1 && (reinterpret_cast<uintptr_t>(a.green) & 15) == 0) {
            constexpr int CH = TX / PER;
            for (int e = threadIdx.x; e < N * CH; e += blockDim.x) {
                const int j = e / CH, ch = e % CH;
                cp_async<16>(gs + j * TX + ch * PER, g + x0 + ch * PER + j * gl);
            }
            cp_async_commit();
            return;
        }
    }
    for (int e = threadIdx.x; e < N * TX; e += blockDim.x) {
        const int j = e / TX, cc = e % TX, xx = x0 + cc;
        if (xx < a.nx) cp_async<sizeof(T)>(gs + e, g + (int64_t)fold_idx(xx, a.f_x) * a.g_x + j * gl);
        else gs[e] = (T)0;
    }
    cp_async_commit();
}

// resident threads per SM the register budget is sized for (2 CTAs of 256
// threads): the passes are bound by memory and issue, and two resident
// CTAs overlap one CTA's loads with the other's arithmetic
#ifndef FLB_COL_THREADS_PER_SM
#define FLB_COL_THREADS_PER_SM 512
#endif
#ifndef FLB_FUSED_THREADS_PER_SM
#define FLB_FUSED_THREADS_PER_SM 512
#endif
// FP64 column passes with a first radix of 32 (and every FP64 fused pass) hold
// 16-32 complex doubles and their twiddles in registers: 256 threads per SM,
// up to 255 registers each, instead of spilling at 128
#ifndef FLB_F64_WIDE_THREADS_PER_SM
#define FLB_F64_WIDE_THREADS_PER_SM 256
#endif
// FP32 forward column passes of power-of-two lines (first radix 32): three
// 256-thread CTAs per SM at 80 registers, the stage table read through L1
// so that three CTAs' exchange lines fit in shared memory
template <typename T, int MODE, int R1>
struct Fwd3 {
    static constexpr bool ON = MODE == 0 && R1 == 32 && sizeof(T) == 4;
};

// FP32 r2c rows of power-of-two length: three CTAs per SM at 80 registers,
// the stage table read through L1 so that three CTAs' lines fit
template <typename T, int R1>
struct Row3 {
    static constexpr bool ON = R1 == 32 && sizeof(T) == 4;
};

template <int THREADS, bool FUSED = false, bool F64_WIDE = false, bool THREE = false>
struct Occ {
    static constexpr int per_sm = THREE ? 768 : (F64_WIDE ? FLB_F64_WIDE_THREADS_PER_SM : (FUSED ? FLB_FUSED_THREADS_PER_SM : FLB_COL_THREADS_PER_SM));
    static constexpr int want = per_sm / (THREADS < 64 ? 64 : THREADS);
    static constexpr int blocks = want < 1 ? 1 : want;
};

// ---------------------------------------------------------------- columns
// Extent of the loaded / stored part of a line, known at compile time:
// tested per element, L/2, L; L/2 + 1 (the zero-padded line of a node-centred
// unbounded direction: n nodes in a 2 (n - 1)-point line; fused passes only)
enum { SH_ANY = 0, SH_HALF = 1, SH_FULL = 2, SH_HALF1 = 3 };
// MODE 0: forward DFT (SH: loaded part; SH != ANY also means all L stored),
//      1: inverse DFT (SH: stored part; SH != ANY also means all L loaded),
//      2: forward, Green multiply, inverse (SH: loaded and stored part).
// The host guarantees L * (line stride) < 2^31 (32-bit offsets along a line).
template <typename T, int L, int R1, int TX, int MODE, int SH>
__global__ void __launch_bounds__(TX * (L / R1), (Occ<TX * (L / R1), MODE == 2, sizeof(T) == 8 && (MODE == 2 || R1 == 32), Fwd3<T, MODE, R1>::ON && TX * (L / R1) == 256>::blocks)) col_dft_kernel(const __grid_constant__ ColArgs a) {
    using F = RegFFT<T, L, R1, false, Fwd3<T, MODE, R1>::ON && TX * (L / R1) == 256>;
    using C = typename CT<T>::C;
    constexpr int INS = (MODE == 1) ? (SH == SH_ANY ? SH_ANY : SH_FULL) : SH;
    constexpr int OUTS = (MODE == 0) ? (SH == SH_ANY ? SH_ANY : SH_FULL) : SH;
    static_assert(SH != SH_HALF1 || MODE == 2, "L/2 + 1 lines are fused passes");
    constexpr bool ZH = INS == SH_HALF || INS == SH_HALF1;
    constexpr int NLD = ZH ? R1 / 2 : R1;  // registers loaded
    constexpr int NST = (OUTS == SH_HALF || OUTS == SH_HALF1) ? R1 / 2 : R1;  // registers stored
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int c = threadIdx.x % TX, p = threadIdx.x / TX;
    const int x = blockIdx.x * TX + c;
    const int o = (MODE == 2) ? mirror_order(blockIdx.y, a.nouter, a.f_outer) : (int)blockIdx.y;
    const int comp = blockIdx.z;
    const bool valid = x < a.nx;
    if constexpr (MODE != 2) prefetch_ahead<false>(a.pf, TX * (int)(sizeof(C) / 8), 0);
    // shared memory: TX lines of the exchange, the stage table, the Green's values
    const C* tws = stage_twiddles<F>(a.tws, sm + TX * F::SC);
    T* gs = reinterpret_cast<T*>(sm + TX * F::SC + F::TW_SMEM);
    if constexpr (MODE == 2) stage_green<T, L, TX>(a, gs, o);
    // lanes outside the array read its first element and drop it (no branch)
    const C* in = valid ? reinterpret_cast<const C*>(a.in) + comp * a.in_cstr + (int64_t)o * a.in_ostr + x + (int64_t)p * a.in_lstr
                        : reinterpret_cast<const C*>(a.in);
    int ls = valid ? F::P * (int)a.in_lstr : 0;
    if constexpr (MODE == 1) {
        if (a.peers.n > 0 && valid) {
            int lstr;
            in = peer_column<C>(a.peers, x, o, p, lstr);
            ls = F::P * lstr;
        }
    }
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        if (r >= NLD) {
            v[r] = mkc((T)0, (T)0);
        } else if constexpr (INS != SH_ANY) {
            // a lane past the last column reads the array's first element: its
            // line (own exchange row, own Green's values) is never stored
            v[r] = in[r * ls];
        } else {
            const bool ok = valid && p + F::P * r < a.nin;
            const C t = in[ok ? r * ls : 0];
            v[r] = ok ? t : mkc((T)0, (T)0);
        }
    }
    // x_{L/2} of an L/2 + 1 line: lane 0's register R1/2
    C xh = mkc((T)0, (T)0);
    if constexpr (INS == SH_HALF1) {
        if (p == 0) xh = in[(R1 / 2) * ls];
    }
    // the table's copies are complete before the first exchange's barrier
    if constexpr (F::TWS) {
        if constexpr (MODE == 2) cp_async_wait<1>();
        else cp_async_wait<0>();
    }
    C* line = sm + c * F::SC;
    if constexpr (MODE == 1) F::template fft<false, true>(v, line, p, tws);
    else F::template fft<ZH, false, INS == SH_HALF1>(v, line, p, tws, xh);
    if constexpr (MODE == 2) {
        cp_async_wait_all();
        __syncthreads();
        // k = p + P r; fold(k) = k for r < R1/2, L - k for r >= R1/2 (k = L/2 included)
        // the stored spectrum already carries the normalisation
        const T* g0 = gs + p * TX + c;
        const T* g1 = gs + (L - p) * TX + c;
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = cscale(v[r], r < R1 / 2 ? g0[r * F::P * TX] : g1[-r * F::P * TX]);
        // the table plus an offset the compiler cannot see is zero: it cannot
        // merge the second DFT's twiddle loads with the first's, so those stay
        // out of registers during the multiply (the state space stays known)
        int zero = 0;
        asm("" : "+r"(zero));
        F::template fft<false, true>(v, line, p, tws + zero);
    }
    if (valid) {
        C* out = reinterpret_cast<C*>(a.out) + comp * a.out_cstr + (int64_t)o * a.out_ostr + x + (int64_t)p * a.out_lstr;
        int os = F::P * (int)a.out_lstr;
        if constexpr (MODE == 0) {
            if (a.peers.n > 0) {
                int lstr;
                out = peer_column<C>(a.peers, x, o, p, lstr);
                os = F::P * lstr;
            }
        }
#pragma unroll
        for (int r = 0; r < NST; ++r) {
            if (OUTS != SH_ANY || p + F::P * r < a.nout) out[r * os] = v[r];
        }
        if constexpr (OUTS == SH_HALF1) {
            if (p == 0) out[(R1 / 2) * os] = v[R1 / 2];
        }
    }
}

// ---------------------------------------------------------------- columns, ROT
// The curl and Green's multiply of a ROT solve fused between the forward and
// inverse DFT of the last direction (dothemagic_rot.ipp:102-350 between the
// transforms of Solver.cpp:1402-1462): the three components of TX columns
// meet in one CTA, one group of TX x P threads per component.  After the
// forward DFT every group puts its spectrum in its own exchange lines, reads
// the other two components at the same wave numbers, forms its component of
// G (i K x w),
//   u_g = G (w_{g+2} K_{g+1,g+2} - w_{g+1} K_{g+2,g+1})  (indices mod 3),
// and transforms it back.  K_{d,c} is read from per-direction tables (the
// spectral or finite-difference symbol with the phase of the derivative);
// along the line it changes with the wave number, along x and the outer
// direction it is one value per thread.
template <typename T, int L>
struct RotTile {
    static constexpr int R1 = fast_radix1_mode(L, sizeof(T) == 8, 2);
    static constexpr int P = L / R1;
    // threads per component group: 128, or 64 for the FP64 lines of first
    // radix 32 (up to 255 registers).  Measured at 384^3 (768-point lines,
    // FP32): 5.90 ms with 128, 6.66 ms with 64 at two CTAs per SM (16-byte
    // row segments)
#ifndef FLB_ROT_GROUP
#define FLB_ROT_GROUP 128
#endif
    static constexpr int GROUP = (sizeof(T) == 8 && R1 == 32) ? FLB_ROT_GROUP / 2 : FLB_ROT_GROUP;
    static constexpr int TX = P >= GROUP ? 1 : GROUP / P;
    static constexpr int THREADS = 3 * TX * P;
};
#ifndef FLB_ROT_MINB
#define FLB_ROT_MINB 1
#endif

template <typename T, int L, int R1, int TX, int SH>
__global__ void __launch_bounds__(3 * TX * (L / R1), FLB_ROT_MINB) col_rot_kernel(const __grid_constant__ ColArgs a) {
    using F = RegFFT<T, L, R1>;
    using C = typename CT<T>::C;
    constexpr int P = F::P, GT = TX * P;
    constexpr int NLD = (SH == SH_HALF) ? R1 / 2 : R1;  // registers loaded
    constexpr int NST = NLD;                             // registers stored
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int g = threadIdx.x / GT, t = threadIdx.x % GT;  // component group; thread in it
    const int c = t % TX, p = t / TX;
    const int x = blockIdx.x * TX + c;
    const int o = mirror_order(blockIdx.y, a.nouter, a.f_outer);
    const int comp = 3 * blockIdx.z + g;
    const bool valid = x < a.nx;
    const C* tws = stage_twiddles<F>(a.tws, sm + 3 * TX * F::SC);
    T* gs = reinterpret_cast<T*>(sm + 3 * TX * F::SC + F::TW_SMEM);
    stage_green<T, L, TX>(a, gs, o);
    // lanes outside the array read its first element and drop it (no branch)
    const C* in = valid ? reinterpret_cast<const C*>(a.in) + comp * a.in_cstr + (int64_t)o * a.in_ostr + x + (int64_t)p * a.in_lstr
                        : reinterpret_cast<const C*>(a.in);
    const int ls = valid ? P * (int)a.in_lstr : 0;
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        if (r >= NLD) {
            v[r] = mkc((T)0, (T)0);
        } else if constexpr (SH != SH_ANY) {
            v[r] = in[r * ls];
        } else {
            const bool ok = valid && p + P * r < a.nin;
            const C u = in[ok ? r * ls : 0];
            v[r] = ok ? u : mkc((T)0, (T)0);
        }
    }
    if constexpr (F::TWS) cp_async_wait<1>();
    C* line = sm + (g * TX + c) * F::SC;
    F::template fft<SH == SH_HALF, false>(v, line, p, tws);
    // the two symbols of this group: K_a = K_{g+1, g+2} multiplies w_{g+2},
    // K_b = K_{g+2, g+1} multiplies w_{g+1}; at most one of them runs along the line
    const int ga = (g + 2) % 3, gb = (g + 1) % 3;
    const C* K = reinterpret_cast<const C*>(a.ksym);
    const int xi = valid ? x : 0;
    auto at = [&](int d) { return d == 0 ? xi : o; };
    const C* ktab = nullptr;
    int vary = 0;  // 1: K_a along the line, 2: K_b along the line
    C ka = mkc((T)0, (T)0), kb = mkc((T)0, (T)0);
    if (gb == a.ax_line) {
        vary = 1;
        ktab = K + (3 * gb + ga) * a.kstr;
    } else {
        ka = K[(3 * gb + ga) * a.kstr + at(gb)];
    }
    if (ga == a.ax_line) {
        vary = 2;
        ktab = K + (3 * ga + gb) * a.kstr;
    } else {
        kb = K[(3 * ga + gb) * a.kstr + at(ga)];
    }
    cp_async_wait_all();
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R1; ++r) line[F::sw(p + P * r)] = v[r];
    __syncthreads();
    {
        const C* fa = sm + (ga * TX + c) * F::SC;
        const C* fb = sm + (gb * TX + c) * F::SC;
        // k = p + P r; fold(k) = k for r < R1/2, L - k above (k = L/2 included);
        // the stored spectrum already carries the normalisation
        const T* g0 = gs + p * TX + c;
        const T* g1 = gs + (L - p) * TX + c;
        auto curl = [&](auto mode) {
            constexpr int VARY = decltype(mode)::value;
#pragma unroll
            for (int r = 0; r < R1; ++r) {
                const int k = p + P * r;
                const C A = (VARY == 1) ? __ldg(ktab + k) : ka;
                const C B = (VARY == 2) ? __ldg(ktab + k) : kb;
                const C u = csub(cmul(fa[F::sw(k)], A), cmul(fb[F::sw(k)], B));
                v[r] = cscale(u, r < R1 / 2 ? g0[r * P * TX] : g1[-r * P * TX]);
            }
        };
        if (vary == 1) curl(std::integral_constant<int, 1>{});
        else if (vary == 2) curl(std::integral_constant<int, 2>{});
        else curl(std::integral_constant<int, 0>{});
    }
    // every group has read the others' spectra before the inverse DFT reuses the lines
    __syncthreads();
    int zero = 0;
    asm("" : "+r"(zero));
    F::template fft<false, true>(v, line, p, tws + zero);
    if (valid) {
        C* out = reinterpret_cast<C*>(a.out) + comp * a.out_cstr + (int64_t)o * a.out_ostr + x + (int64_t)p * a.out_lstr;
        const int os = P * (int)a.out_lstr;
#pragma unroll
        for (int r = 0; r < NST; ++r) {
            if (SH != SH_ANY || p + P * r < a.nout) out[r * os] = v[r];
        }
    }
}

// ---------------------------------------------------------------- rows: fused
// Last-direction pass along x: rows are contiguous, so a row belongs to P
// consecutive lanes of one warp (P = L / R1 <= 32) and every exchange of its
// register DFTs synchronises the warp only; warps run independently.  The
// row's folded Green's values (L/2 + 1, x folded at L) arrive in the line's
// shared memory through cp.async while the row loads and the forward DFT run.
// SH: loaded and stored part (SH_HALF: the zero-padded half is neither loaded
// nor computed, the truncated half neither computed nor stored).
template <typename T, int L>
struct RowFusedTile {
    static constexpr int GP = ((L / 2 + 1) * (int)sizeof(T) + 15) / 16 * 16 / (int)sizeof(T);  // Green's values staged per row
};

// Register budget: 384 threads per SM in FP32 (up to 170 registers; 512,
// at 128 registers with a few spilled, ran 1.39 against 1.28 ms for the
// 1024-point rows of a 512^3 solve), 256 in FP64 (up to 255 registers)
#ifndef FLB_ROWF_WARPS
#define FLB_ROWF_WARPS 4
#endif
template <typename T>
struct RowFusedOcc {
    static constexpr int per_sm = sizeof(T) == 8 ? 256 : 384;
    static constexpr int blocks = per_sm / (FLB_ROWF_WARPS * 32) > 0 ? per_sm / (FLB_ROWF_WARPS * 32) : 1;
};

template <typename T, int L, int R1, int WARPS, int SH>
__global__ void __launch_bounds__(WARPS * 32, RowFusedOcc<T>::blocks) row_fused_kernel(const __grid_constant__ RowFusedArgs a) {
    using F = RegFFT<T, L, R1, true, true, true>;
    using C = typename CT<T>::C;
    constexpr int P = F::P, LPW = 32 / P, GP = RowFusedTile<T, L>::GP;
    constexpr int NLD = (SH == SH_HALF) ? R1 / 2 : R1;
    constexpr int NST = NLD;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = lane % P, li = warp * LPW + lane / P;  // line of the CTA
    const int64_t row = (int64_t)blockIdx.x * (WARPS * LPW) + li;
    const int comp = blockIdx.y;
    const bool valid = row < (int64_t)a.n1 * a.n2;
    const int i1 = valid ? (int)(row % a.n1) : 0, i2 = valid ? (int)(row / a.n1) : 0;
    C* line = sm + li * F::SC;
    T* gs = reinterpret_cast<T*>(sm + WARPS * LPW * F::SC) + li * GP;
    {
        const T* g = reinterpret_cast<const T*>(a.green) + (int64_t)fold_idx(i1, a.f1) * a.g1 + (int64_t)fold_idx(i2, a.f2) * a.g2;
        constexpr int PER = 16 / (int)sizeof(T), CH = GP / PER;
        for (int e = p; e < CH; e += P) cp_async<16>(gs + e * PER, g + e * PER);
        cp_async_commit();
    }
    const C* in = reinterpret_cast<const C*>(a.in) + comp * a.cstr + (int64_t)i1 * a.s1 + (int64_t)i2 * a.s2 + p;
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        if (r >= NLD) {
            v[r] = mkc((T)0, (T)0);
        } else if constexpr (SH != SH_ANY) {
            v[r] = in[P * r];
        } else {
            const bool ok = p + P * r < a.nin;
            const C u = in[ok ? P * r : 0];
            v[r] = ok ? u : mkc((T)0, (T)0);
        }
    }
    const C* tws = reinterpret_cast<const C*>(a.tws);
    F::template fft<SH == SH_HALF, false>(v, line, p, tws);
    cp_async_wait_all();
    __syncwarp();
    // k = p + P r; fold(k) = k for r < R1/2, L - k above; the stored spectrum carries the normalisation
#pragma unroll
    for (int r = 0; r < R1; ++r) v[r] = cscale(v[r], r < R1 / 2 ? gs[p + P * r] : gs[L - p - P * r]);
    int zero = 0;
    asm("" : "+r"(zero));
    F::template fft<false, true>(v, line, p, tws + zero);
    if (valid) {
        C* out = reinterpret_cast<C*>(a.out) + comp * a.cstr + (int64_t)i1 * a.s1 + (int64_t)i2 * a.s2 + p;
#pragma unroll
        for (int r = 0; r < NST; ++r) {
            if (SH != SH_ANY || p + P * r < a.nout) out[P * r] = v[r];
        }
    }
}

// ROT along x rows: warps in triples, warp g of a triple holding component g
// of LPW row positions; after the forward DFT the three warps of a triple
// meet at a named barrier (no other warp waits) to read each other's spectra
// for the curl, as in col_rot_kernel.
//
// With x last, z is the real-to-complex direction, and the spectrum kept is
// kz <= N instead of the reference's kx <= N.  An odd derivative is not
// Hermitian at a Nyquist index (its symbol there equals that of the negated
// index), so the two orders would discard different parts of the curl in
// their final complex-to-real transform.  The row kernel therefore forms the
// reference's spectrum: the curl with the symbols at +k (P) for 0 < kx < N,
// the conjugate of the curl at -k (Q = conj of the symbols at -k, which is
// the symbol at k with its sign flipped except at a Nyquist index) for
// kx > N, and (P + Q) / 2 at kx = 0 and kx = N (the reference's x
// complex-to-real keeps the real part there).
#ifndef FLB_ROWROT_TRIPLES
#define FLB_ROWROT_TRIPLES 2
#endif

template <typename T, int L, int R1, int NT, int SH>
__global__ void __launch_bounds__(NT * 96, RowFusedOcc<T>::per_sm / (NT * 96) > 0 ? RowFusedOcc<T>::per_sm / (NT * 96) : 1)
    row_rot_kernel(const __grid_constant__ RowFusedArgs a) {
    using F = RegFFT<T, L, R1, true, true, true>;
    using C = typename CT<T>::C;
    constexpr int P = F::P, LPW = 32 / P, GP = RowFusedTile<T, L>::GP;
    constexpr int NLD = (SH == SH_HALF) ? R1 / 2 : R1;
    constexpr int NST = NLD;
    static_assert(NT >= 1 && NT <= 15, "named barriers 1..15");
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tri = warp / 3, g = warp % 3;
    const int p = lane % P, lw = lane / P;
    const int64_t row = (int64_t)blockIdx.x * (NT * LPW) + tri * LPW + lw;  // row position
    const bool valid = row < (int64_t)a.n1 * a.n2;
    if (a.pf.nbox > 0 && threadIdx.x == 0) {
        // the rows of the block pf.dist launches ahead (x, then y order), into L2
        const long long lin = blockIdx.x + (long long)gridDim.x * blockIdx.y + a.pf.dist;
        const int bx = (int)(lin % gridDim.x), by = (int)(lin / gridDim.x);
        if (by < (int)gridDim.y) {
            const int64_t row0 = (int64_t)bx * (NT * LPW);
            const int p1 = (int)(row0 % a.n1), p2 = (int)(row0 / a.n1);
            for (int gg = 0; gg < 3; ++gg)
                for (int k = 0; k < a.pf.nbox; ++k) l2_prefetch_box(&a.pf.map, k * a.pf.step, p1, p2, 3 * by + gg);
        }
    }
    const int i1 = valid ? (int)(row % a.n1) : 0, i2 = valid ? (int)(row / a.n1) : 0;
    const int comp = 3 * blockIdx.y + g;
    // lines of the triple: [component][lw]; Green's rows of the triple after all lines
    auto line_of = [&](int gg) { return sm + ((tri * 3 + gg) * LPW + lw) * F::SC; };
    C* line = line_of(g);
    T* gs = reinterpret_cast<T*>(sm + NT * 3 * LPW * F::SC) + (tri * LPW + lw) * GP;
    if (g == 0) {
        const T* gr = reinterpret_cast<const T*>(a.green) + (int64_t)fold_idx(i1, a.f1) * a.g1 + (int64_t)fold_idx(i2, a.f2) * a.g2;
        constexpr int PER = 16 / (int)sizeof(T), CH = GP / PER;
        for (int e = p; e < CH; e += P) cp_async<16>(gs + e * PER, gr + e * PER);
        cp_async_commit();
    }
    const C* in = reinterpret_cast<const C*>(a.in) + comp * a.cstr + (int64_t)i1 * a.s1 + (int64_t)i2 * a.s2 + p;
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        if (r >= NLD) {
            v[r] = mkc((T)0, (T)0);
        } else if constexpr (SH != SH_ANY) {
            v[r] = in[P * r];
        } else {
            const bool ok = p + P * r < a.nin;
            const C u = in[ok ? P * r : 0];
            v[r] = ok ? u : mkc((T)0, (T)0);
        }
    }
    const C* tws = reinterpret_cast<const C*>(a.tws);
    F::template fft<SH == SH_HALF, false>(v, line, p, tws);
    // the curl terms of component g: K_a = K_{g+1, g+2} w_{g+2} - K_b = K_{g+2, g+1} w_{g+1};
    // x (the line) is direction 0, i1 and i2 are directions a.ax1 and a.ax2
    const int ga = (g + 2) % 3, gb = (g + 1) % 3;
    const C* K = reinterpret_cast<const C*>(a.ksym);
    auto at = [&](int d) { return d == a.ax1 ? i1 : i2; };
    const C* ktab = nullptr;
    int vary = 0;
    C ka = mkc((T)0, (T)0), kb = mkc((T)0, (T)0);
    // sign of the symbol at the negated index, for the symbols constant along the row
    T sa = (T)-1, sb = (T)-1;
    if (gb == 0) {
        vary = 1;
        ktab = K + (3 * gb + ga) * a.kstr;
    } else {
        ka = K[(3 * gb + ga) * a.kstr + at(gb)];
        if (at(gb) == a.nyq[gb]) sa = (T)1;
    }
    if (ga == 0) {
        vary = 2;
        ktab = K + (3 * ga + gb) * a.kstr;
    } else {
        kb = K[(3 * ga + gb) * a.kstr + at(ga)];
        if (at(ga) == a.nyq[ga]) sb = (T)1;
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R1; ++r) line[F::sw(p + P * r)] = v[r];
    if (g == 0) cp_async_wait_all();
    asm volatile("bar.sync %0, 96;" ::"r"(1 + tri) : "memory");
    {
        const C* fa = line_of(ga);
        const C* fb = line_of(gb);
        {
            // one code path for the three components of the triple (which
            // symbol varies along the row is a per-warp value): three unrolled
            // variants, one per component, missed the instruction cache
            // (fused rows 3.05 -> 2.94 ms at 384^3)
            const bool v1 = vary == 1, v2 = vary == 2;
            const C* kt = ktab ? ktab : K;
            // the Q form's symbols: the constant ones (sign times conjugate)
            // once per lane; the varying one is -conj(kv), conj(kv) at kx = N
            const C qka = mkc(sa * ka.x, -sa * ka.y), qkb = mkc(sb * kb.x, -sb * kb.y);
#pragma unroll
            for (int r = 0; r < R1; ++r) {
                const int k = p + P * r;
                const C kv = vary ? __ldg(kt + k) : mkc((T)0, (T)0);
                const C A = v1 ? kv : ka;
                const C B = v2 ? kv : kb;
                const C wa = fa[F::sw(k)], wb = fb[F::sw(k)];
                C u = csub(cmul(wa, A), cmul(wb, B));
                if (r >= R1 / 2 || (r == 0 && p == 0)) {
                    const bool edge = (p == 0) && (r == 0 || r == R1 / 2);
                    const C qv = (p == 0 && r == R1 / 2) ? mkc(kv.x, -kv.y) : mkc(-kv.x, kv.y);
                    const C q = csub(cmul(wa, v1 ? qv : qka), cmul(wb, v2 ? qv : qkb));
                    u = edge ? mkc((T)0.5 * (u.x + q.x), (T)0.5 * (u.y + q.y)) : q;
                }
                v[r] = cscale(u, r < R1 / 2 ? gs[k] : gs[L - k]);
            }
        }
    }
    // the triple has read every spectrum before the inverse DFT reuses the lines
    asm volatile("bar.sync %0, 96;" ::"r"(1 + tri) : "memory");
    int zero = 0;
    asm("" : "+r"(zero));
    F::template fft<false, true>(v, line, p, tws + zero);
    if (valid) {
        C* out = reinterpret_cast<C*>(a.out) + comp * a.cstr + (int64_t)i1 * a.s1 + (int64_t)i2 * a.s2 + p;
#pragma unroll
        for (int r = 0; r < NST; ++r) {
            if (SH != SH_ANY || p + P * r < a.nout) out[P * r] = v[r];
        }
    }
}

template <typename T, int L, int NT, int SH>
inline cudaError_t launch_row_rot_t(const RowFusedArgs& a, int ncomp, cudaStream_t s) {
    constexpr int R1 = fast_radix1_rowrot(L, sizeof(T) == 8);
    using F = RegFFT<T, L, R1, true, true, true>;
    constexpr int LPW = 32 / F::P;
    constexpr size_t smem = (size_t)NT * LPW * (3 * F::SC * sizeof(typename CT<T>::C) + RowFusedTile<T, L>::GP * sizeof(T));
    static_assert(smem <= 227 * 1024, "row tile too large");
    if (ncomp % 3 != 0 || a.g1 < RowFusedTile<T, L>::GP || (reinterpret_cast<uintptr_t>(a.green) & 15) != 0 ||
        (a.g1 * sizeof(T)) % 16 != 0 || (a.g2 * sizeof(T)) % 16 != 0)
        return cudaErrorInvalidValue;
    static std::atomic<unsigned long long> attr{0};
    if (cudaError_t e = smem_attr_once(attr, row_rot_kernel<T, L, R1, NT, SH>, smem); e != cudaSuccess) return e;
    const int64_t rows = (int64_t)a.n1 * a.n2;
    dim3 grid((unsigned)((rows + NT * LPW - 1) / (NT * LPW)), ncomp / 3);
    row_rot_kernel<T, L, R1, NT, SH><<<grid, NT * 96, smem, s>>>(a);
    return cudaGetLastError();
}

// lines of first radix R1 whose P = L / R1 threads fit in one warp
__host__ __device__ constexpr bool fast_rowfused_len(int L, int f64) {
    return (L == 48 || L == 64 || L == 96 || L == 128 || L == 192 || L == 256 || L == 384 || L == 512 || L == 768 || L == 1024) &&
           L / fast_radix1_rowfused(L, f64) <= 32;
}

template <typename T, int L, int WARPS, int SH>
inline cudaError_t launch_row_fused_t(const RowFusedArgs& a, int ncomp, cudaStream_t s) {
    constexpr int R1 = fast_radix1_rowfused(L, sizeof(T) == 8);
    using F = RegFFT<T, L, R1, true, true, true>;
    constexpr int LPW = 32 / F::P;
    constexpr size_t smem = (size_t)WARPS * LPW * (F::SC * sizeof(typename CT<T>::C) + RowFusedTile<T, L>::GP * sizeof(T));
    static_assert(smem <= 227 * 1024, "row tile too large");
    if (a.g1 < RowFusedTile<T, L>::GP || (reinterpret_cast<uintptr_t>(a.green) & 15) != 0 || (a.g1 * sizeof(T)) % 16 != 0 ||
        (a.g2 * sizeof(T)) % 16 != 0)
        return cudaErrorInvalidValue;
    static std::atomic<unsigned long long> attr{0};
    if (cudaError_t e = smem_attr_once(attr, row_fused_kernel<T, L, R1, WARPS, SH>, smem); e != cudaSuccess) return e;
    const int64_t rows = (int64_t)a.n1 * a.n2;
    dim3 grid((unsigned)((rows + WARPS * LPW - 1) / (WARPS * LPW)), ncomp);
    row_fused_kernel<T, L, R1, WARPS, SH><<<grid, WARPS * 32, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename T, int SH, bool ROT>
inline cudaError_t launch_row_fused_len(int L, const RowFusedArgs& a, int ncomp, cudaStream_t s) {
    constexpr int f64 = sizeof(T) == 8;
    switch (L) {
#define FLB_ROWF_CASE(n)                                                                        \
    case n:                                                                                     \
        if constexpr (fast_rowfused_len(n, f64)) {                                              \
            if constexpr (ROT) return launch_row_rot_t<T, n, FLB_ROWROT_TRIPLES, SH>(a, ncomp, s); \
            else return launch_row_fused_t<T, n, FLB_ROWF_WARPS, SH>(a, ncomp, s);              \
        }                                                                                       \
        break;
        FLB_ROWF_CASE(48)
        FLB_ROWF_CASE(64)
        FLB_ROWF_CASE(96)
        FLB_ROWF_CASE(128)
        FLB_ROWF_CASE(192)
        FLB_ROWF_CASE(256)
        FLB_ROWF_CASE(384)
        FLB_ROWF_CASE(512)
        FLB_ROWF_CASE(768)
        FLB_ROWF_CASE(1024)
#undef FLB_ROWF_CASE
    }
    return cudaErrorInvalidValue;
}

template <typename T, bool ROT>
inline cudaError_t launch_row_fused_shape(int sh, int L, const RowFusedArgs& a, int ncomp, cudaStream_t s) {
    if (sh == SH_FULL) return launch_row_fused_len<T, SH_FULL, ROT>(L, a, ncomp, s);
    if (sh == SH_HALF) return launch_row_fused_len<T, SH_HALF, ROT>(L, a, ncomp, s);
    return launch_row_fused_len<T, SH_ANY, ROT>(L, a, ncomp, s);
}

// CTAs per SM the real-side columns ask the compiler for: three for FP32
// real-to-complex lines of a first radix up to 24 (80 registers; 384^3 ROT z
// forward 0.568 -> 0.514 ms; the complex-to-real lines and the radix-32
// lines were slower so), else the column passes' figure;
// FLB_COLREAL_PER_SM > 0 sets threads per SM for all of them
#ifndef FLB_COLREAL_PER_SM
#define FLB_COLREAL_PER_SM 0
#endif
template <typename T, int R1, bool C2R, int THREADS>
struct ColRealOcc {
    static constexpr int dflt = (sizeof(T) == 4 && R1 <= 16 && THREADS == 256)
                                    ? 4
                                    : ((sizeof(T) == 4 && !C2R && R1 <= 24 && THREADS == 256) ? 3 : Occ<THREADS>::blocks);
    static constexpr int blocks =
        FLB_COLREAL_PER_SM > 0 ? (FLB_COLREAL_PER_SM / THREADS > 0 ? FLB_COLREAL_PER_SM / THREADS : 1) : dflt;
};

// ---------------------------------------------------------------- columns, real side
// r2c (C2R = false): real column of nin values (zero beyond) -> X[0..L/2];
// SH: loaded part.  c2r (C2R = true): X[0..L/2] -> real column, the upper half
// of the spectrum read as conj(X[L-k]) straight from memory (no exchange);
// SH: stored part.  Im X[0] and Im X[L/2] do not enter a real result.
// RT: type of the real side (the working precision, or the user's doubles
// when the pass is the first or last of a solve).
template <typename T, typename RT, int L, int R1, int TX, bool C2R, int SH>
__global__ void __launch_bounds__(TX * (L / R1), ColRealOcc<T, R1, C2R, TX * (L / R1)>::blocks) col_real_kernel(const ColArgs a) {
    using F = RegFFT<T, L, R1>;
    using C = typename CT<T>::C;
    constexpr int P = F::P;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int c = threadIdx.x % TX, p = threadIdx.x / TX;
    const int x = blockIdx.x * TX + c;
    const int o = blockIdx.y;
    const int comp = blockIdx.z;
    const bool valid = x < a.nx;
    const C* tws = stage_twiddles<F>(a.tws, sm + TX * F::SC);
    C v[R1];
    if constexpr (!C2R) {
        constexpr int NLD = (SH == SH_HALF) ? R1 / 2 : R1;
        const RT* in = valid ? reinterpret_cast<const RT*>(a.in) + comp * a.in_cstr + (int64_t)o * a.in_ostr + x + (int64_t)p * a.in_lstr
                             : reinterpret_cast<const RT*>(a.in);
        const int ls = valid ? P * (int)a.in_lstr : 0;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            if (r >= NLD) {
                v[r] = mkc((T)0, (T)0);
            } else {
                const bool ok = valid && (SH != SH_ANY || p + P * r < a.nin);
                const RT t = in[ok ? r * ls : 0];
                v[r] = mkc(ok ? (T)t : (T)0, (T)0);
            }
        }
    } else {
        // X[k] for k <= L/2 (r < R1/2, and r = R1/2 on p = 0); conj X[L-k] above
        const C* base = valid ? reinterpret_cast<const C*>(a.in) + comp * a.in_cstr + (int64_t)o * a.in_ostr + x
                              : reinterpret_cast<const C*>(a.in);
        const int lstr = valid ? (int)a.in_lstr : 0;
        const C* lo = base + (int64_t)p * lstr;
        const C* hi = base + (int64_t)(L - p) * lstr;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            C t;
            if (r < R1 / 2) t = lo[r * P * lstr];
            else t = cconj(hi[-r * P * lstr]);  // k = L/2 (r = R1/2, p = 0): conj X[L/2], imaginary part dropped below
            if (r == 0 && p == 0) t.y = (T)0;
            if (r == R1 / 2 && p == 0) t.y = (T)0;
            v[r] = valid ? t : mkc((T)0, (T)0);
        }
    }
    if constexpr (F::TWS) cp_async_wait<0>();
    C* line = sm + c * F::SC;
    if constexpr (C2R) F::template fft<false, true>(v, line, p, tws);
    else F::template fft<SH == SH_HALF, false>(v, line, p, tws);
    if (!valid) return;
    if constexpr (!C2R) {
        C* out = reinterpret_cast<C*>(a.out) + comp * a.out_cstr + (int64_t)o * a.out_ostr + x + (int64_t)p * a.out_lstr;
        const int os = P * (int)a.out_lstr;
#pragma unroll
        for (int r = 0; r <= R1 / 2; ++r) {
            if (r < R1 / 2 || p == 0) out[r * os] = v[r];
        }
        if (p == 0 && a.period >= 0) out[(int64_t)a.period * a.out_lstr] = v[0];
    } else {
        constexpr int NST = (SH == SH_HALF) ? R1 / 2 : R1;
        RT* out = reinterpret_cast<RT*>(a.out) + comp * a.out_cstr + (int64_t)o * a.out_ostr + x + (int64_t)p * a.out_lstr;
        const int os = P * (int)a.out_lstr;
#pragma unroll
        for (int r = 0; r < NST; ++r) {
            if (SH != SH_ANY || p + P * r < a.nout) out[r * os] = (RT)v[r].x;
        }
        if (p == 0 && a.period >= 0) out[(int64_t)a.period * a.out_lstr] = (RT)v[0].x;
    }
}

// ---------------------------------------------------------------- columns, real side, in pairs
// The same transforms for two neighbouring columns (x, x + 1) at once: one
// complex DFT of z = a + i b.  r2c: A_k = (Z_k + conj Z_{L-k}) / 2 and
// B_k = (Z_k - conj Z_{L-k}) / 2i, for k <= L/2 (Z_{L-k} from the line in
// shared memory); c2r: Z_k = A_k + i B_k with A_{L-k} = conj A_k (both halves
// read straight from memory), one inverse DFT, a = Re z, b = Im z.  Half the
// arithmetic of one DFT per column, and every global access moves a pair:
// 16 bytes of the real side (doubles) or of the complex side (FP32).  The
// host requires the pairs to be aligned (even strides, aligned base); an odd
// last column is the pair's first half alone.
template <typename T>
struct CPair {
    using C = typename CT<T>::C;
    __device__ static __forceinline__ void ld(const C* p, C& a, C& b) {
        if constexpr (sizeof(T) == 4) {
            const float4 q = *reinterpret_cast<const float4*>(p);
            a = make_float2(q.x, q.y);
            b = make_float2(q.z, q.w);
        } else {
            a = p[0];
            b = p[1];
        }
    }
    __device__ static __forceinline__ void st(C* p, C a, C b) {
        if constexpr (sizeof(T) == 4) {
            *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
        } else {
            p[0] = a;
            p[1] = b;
        }
    }
};

template <typename T, typename RT, int L, int R1, int TXP, bool C2R, int SH>
__global__ void __launch_bounds__(TXP * (L / R1), ColRealOcc<T, R1, C2R, TXP * (L / R1)>::blocks) col_real_pair_kernel(const ColArgs a) {
    using F = RegFFT<T, L, R1>;
    using C = typename CT<T>::C;
    using R2 = typename Vec2<RT>::V;
    constexpr int P = F::P;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int c = threadIdx.x % TXP, p = threadIdx.x / TXP;
    const int x = 2 * (blockIdx.x * TXP + c);  // first column of the pair
    const int o = blockIdx.y;
    const int comp = blockIdx.z;
    const bool valid = x < a.nx, two = x + 1 < a.nx;
    const C* tws = stage_twiddles<F>(a.tws, sm + TXP * F::SC);
    C* line = sm + c * F::SC;
    C v[R1];
    const T z = (T)0;
    if constexpr (!C2R) {
        constexpr int NLD = (SH == SH_HALF) ? R1 / 2 : R1;
        const RT* in = valid ? reinterpret_cast<const RT*>(a.in) + comp * a.in_cstr + (int64_t)o * a.in_ostr + x + (int64_t)p * a.in_lstr
                             : reinterpret_cast<const RT*>(a.in);
        const int ls = valid ? P * (int)a.in_lstr : 0;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            if (r >= NLD) {
                v[r] = mkc(z, z);
            } else {
                const bool ok = valid && (SH != SH_ANY || p + P * r < a.nin);
                if (two) {
                    const R2 t = *reinterpret_cast<const R2*>(in + (ok ? r * ls : 0));
                    v[r] = ok ? mkc((T)t.x, (T)t.y) : mkc(z, z);
                } else {
                    const RT t = in[ok ? r * ls : 0];
                    v[r] = mkc(ok ? (T)t : z, z);
                }
            }
        }
        if constexpr (F::TWS) cp_async_wait<0>();
        F::template fft<SH == SH_HALF, false>(v, line, p, tws);
        // Z_{L-k} from the line: every thread's spectrum in shared memory
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R1; ++r) line[F::sw(p + P * r)] = v[r];
        __syncthreads();
        if (!valid) return;
        C* out = reinterpret_cast<C*>(a.out) + comp * a.out_cstr + (int64_t)o * a.out_ostr + x + (int64_t)p * a.out_lstr;
        const int os = P * (int)a.out_lstr;
        auto split = [&](C zk, int k, C& A, C& B) {
            const C zm = cconj(line[F::sw(k == 0 ? 0 : L - k)]);
            A = mkc((T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y + zm.y));
            B = mkc((T)0.5 * (zk.y - zm.y), (T)-0.5 * (zk.x - zm.x));  // (Z_k - conj Z_{L-k}) / 2i
        };
#pragma unroll
        for (int r = 0; r <= R1 / 2; ++r) {
            if (r < R1 / 2 || p == 0) {
                C A, B;
                split(v[r], p + P * r, A, B);
                if (two) CPair<T>::st(out + r * os, A, B);
                else out[r * os] = A;
            }
        }
        if (p == 0 && a.period >= 0) {
            C A, B;
            split(v[0], 0, A, B);
            C* q = out + (int64_t)a.period * a.out_lstr;
            if (two) CPair<T>::st(q, A, B);
            else *q = A;
        }
    } else {
        // Z_k = A_k + i B_k; for k > L/2 from conj A_{L-k}, conj B_{L-k}
        const C* base = valid ? reinterpret_cast<const C*>(a.in) + comp * a.in_cstr + (int64_t)o * a.in_ostr + x
                              : reinterpret_cast<const C*>(a.in);
        const int lstr = valid ? (int)a.in_lstr : 0;
        const C* lo = base + (int64_t)p * lstr;
        const C* hi = base + (int64_t)(L - p) * lstr;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            C A, B = mkc(z, z);
            const C* q = (r < R1 / 2) ? lo + r * P * lstr : hi - r * P * lstr;
            if (two) CPair<T>::ld(q, A, B);
            else A = *q;
            // Im A_0, Im B_0 and Im A_{L/2}, Im B_{L/2} do not enter real results
            if ((r == 0 || r == R1 / 2) && p == 0) {
                A.y = z;
                B.y = z;
            }
            if (r >= R1 / 2) {
                A = cconj(A);
                B = cconj(B);
            }
            v[r] = valid ? mkc(A.x - B.y, A.y + B.x) : mkc(z, z);
        }
        if constexpr (F::TWS) cp_async_wait<0>();
        F::template fft<false, true>(v, line, p, tws);
        if (!valid) return;
        constexpr int NST = (SH == SH_HALF) ? R1 / 2 : R1;
        RT* out = reinterpret_cast<RT*>(a.out) + comp * a.out_cstr + (int64_t)o * a.out_ostr + x + (int64_t)p * a.out_lstr;
        const int os = P * (int)a.out_lstr;
#pragma unroll
        for (int r = 0; r < NST; ++r) {
            if (SH != SH_ANY || p + P * r < a.nout) {
                if (two) *reinterpret_cast<R2*>(out + r * os) = R2{(RT)v[r].x, (RT)v[r].y};
                else out[r * os] = (RT)v[r].x;
            }
        }
        if (p == 0 && a.period >= 0) {
            RT* q = out + (int64_t)a.period * a.out_lstr;
            if (two) *reinterpret_cast<R2*>(q) = R2{(RT)v[0].x, (RT)v[0].y};
            else *q = (RT)v[0].x;
        }
    }
}

// rows per CTA of the r2c / c2r row kernels: 256 threads, or 128 for the FP64
// rows with a first radix of 32 (255 registers, two CTAs per SM)
template <typename T, int LH, int R1>
struct RowTiles {
    static constexpr bool WIDE = sizeof(T) == 8 && R1 == 32;
    static constexpr int P = LH / R1;
    static constexpr int THREADS = WIDE ? 128 : 256;
    static constexpr int TR = (P >= THREADS) ? 1 : THREADS / P;
};

// ---------------------------------------------------------------- rows: r2c

// IT: type of the real input (the user's double array, or the working precision);
// HALF: nin = Lh (the row is zero-padded to twice its length)
template <typename T, typename IT, int LH, int R1, int TR, bool HALF>
__global__ void __launch_bounds__(TR * (LH / R1), (Occ<TR * (LH / R1), false, RowTiles<T, LH, R1>::WIDE, Row3<T, R1>::ON>::blocks)) row_r2c_kernel(const __grid_constant__ RowArgs a) {
    using F = RegFFT<T, LH, R1, true, Row3<T, R1>::ON>;
    using C = typename CT<T>::C;
    using V = typename Vec2<IT>::V;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int p = threadIdx.x % F::P, rr = threadIdx.x / F::P;
    const int row = blockIdx.x * TR + rr;
    const int comp = blockIdx.y;
    const bool valid = row < a.nrows;
    const int i1 = valid ? row % a.n1 : 0, i2 = valid ? row / a.n1 : 0;
    prefetch_ahead<true>(a.pf, TR, a.n1);
    // rows past the end read the array's first elements and drop them (no branch)
    const IT* src = valid ? reinterpret_cast<const IT*>(a.in) + comp * a.in_cstr + (int64_t)i1 * a.in_s1 + (int64_t)i2 * a.in_s2 + 2 * p
                          : reinterpret_cast<const IT*>(a.in);
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int j = p + F::P * r;
        if (HALF && r >= R1 / 2) {
            v[r] = mkc((T)0, (T)0);
        } else if (HALF) {
            const V d = *reinterpret_cast<const V*>(src + 2 * F::P * r);
            v[r] = valid ? mkc((T)d.x, (T)d.y) : mkc((T)0, (T)0);
        } else {
            const bool two = valid && 2 * j + 1 < a.nin, one = valid && 2 * j + 1 == a.nin;
            const V d = *reinterpret_cast<const V*>(src + (two ? 2 * F::P * r : 0));
            const IT s1 = src[one ? 2 * F::P * r : 0];
            v[r] = two ? mkc((T)d.x, (T)d.y) : (one ? mkc((T)s1, (T)0) : mkc((T)0, (T)0));
        }
    }
    const C* tws = stage_twiddles<F>(a.tws, sm + TR * F::SC);
    C* wsm = sm + TR * F::SC + F::TW_SMEM;
    if constexpr (RowTw<T, LH>::SM) {
        stage_table_part<C, LH>(a.tw, wsm);
        cp_async_commit();
    }
    if constexpr (F::TWS) cp_async_wait<RowTw<T, LH>::SM ? 1 : 0>();
    C* line = sm + rr * F::SC;
    F::template fft<HALF, false>(v, line, p, tws);
    // X[k] = 1/2 (Z_k + conj Z_{LH-k}) - i/2 W_L^k (Z_k - conj Z_{LH-k}),  Z_LH = Z_0
    if constexpr (RowTw<T, LH>::SM) cp_async_wait<0>();
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R1; ++r) line[F::sw(p + F::P * r)] = v[r];
    __syncthreads();
    if (valid) {
        C* dst = reinterpret_cast<C*>(a.out) + comp * a.out_cstr + (int64_t)i1 * a.out_s1 + (int64_t)i2 * a.out_s2 + p;
        const C* tw = (RowTw<T, LH>::SM ? wsm : reinterpret_cast<const C*>(a.tw)) + p;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = p + F::P * r;
            if (k >= a.nout) continue;
            const C zk = v[r];
            const C zm = cconj(line[F::sw(k == 0 ? 0 : LH - k)]);
            const C e = cadd(zk, zm);
            const C d = csub(zk, zm);
            const C w = cmul(tw[F::P * r], d);  // W_L^k (Z_k - conj Z_{LH-k})
            dst[F::P * r] = mkc((T)0.5 * (e.x + w.y), (T)0.5 * (e.y - w.x));
        }
        if (p == 0 && LH < a.nout) {
            const C z0 = line[0];
            dst[LH] = mkc(z0.x - z0.y, (T)0);
        }
    }
}

// ---------------------------------------------------------------- rows: r2r
// DCT / DST I-IV of real rows through the M-point complex DFT of the extended
// row (the general line pass's formulas, csrc/line_pass.cu): the raw row is
// staged in shared memory, c[m] is built from it (reflections, pre-twiddles),
// one forward register DFT, C is exchanged through shared memory for the
// shifted reads of the odd kinds, and Y_k (post-twiddles, post-processing) is
// stored.  IT / OT: types of the real input / output (user doubles or the
// working precision).
template <typename T, typename IT, typename OT, int M, int R1, int TR>
__global__ void __launch_bounds__(TR * (M / R1), (Occ<TR * (M / R1)>::blocks)) row_r2r_kernel(const RowArgs a) {
    using F = RegFFT<T, M, R1, true>;
    using C = typename CT<T>::C;
    constexpr int P = F::P;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int p = threadIdx.x % P, rr = threadIdx.x / P;
    const int row = blockIdx.x * TR + rr;
    const int comp = blockIdx.y;
    const bool valid = row < a.nrows;
    const int i1 = valid ? row % a.n1 : 0, i2 = valid ? row / a.n1 : 0;
    const IT* src = reinterpret_cast<const IT*>(a.in) + comp * a.in_cstr + (int64_t)i1 * a.in_s1 + (int64_t)i2 * a.in_s2;
    C* line = sm + rr * F::SC;
    const C* tws = stage_twiddles<F>(a.tws, sm + TR * F::SC);
    const C* tw = reinterpret_cast<const C*>(a.tw2);
    const int n = a.n, kind = a.kind, nsrc = a.nin;
    const T z = (T)0;
    // raw row in shared memory (zero beyond the source)
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int j = p + P * r;
        const IT u = (valid && j < nsrc) ? src[j] : (IT)0;
        line[F::sw(j)] = mkc((T)u, z);
    }
    if constexpr (F::TWS) cp_async_wait<0>();
    __syncthreads();
    auto u = [&](int t) { return line[F::sw(t)].x; };
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int m = p + P * r;
        T x;
        C c = mkc(z, z);
        switch (kind) {
            case LK_DCT1: c = mkc(m < n ? u(m) : u(M - m), z); break;
            case LK_DST1:
                if (m != 0 && m != n + 1) c = mkc(m <= n ? u(m - 1) : -u(M - m - 1), z);
                break;
            case LK_DCT2: c = mkc(m < n ? u(m) : u(2 * n - 1 - m), z); break;
            case LK_DST2: c = mkc(m < n ? u(m) : -u(2 * n - 1 - m), z); break;
            case LK_DCT3:
                if (m < n) {
                    x = (m == 0 ? (T)1 : (T)2) * u(m);
                    const C w = tw[m];
                    c = mkc(w.x * x, w.y * x);
                }
                break;
            case LK_DST3:
                if (m != 0 && m <= n) {
                    x = (m - 1 == n - 1 ? (T)1 : (T)2) * u(m - 1);
                    const C w = tw[m];
                    c = mkc(w.x * x, w.y * x);
                }
                break;
            default:  // DCT4, DST4
                if (m < n) {
                    x = u(m);
                    const C w = tw[m];
                    c = mkc(w.x * x, w.y * x);
                }
                break;
        }
        v[r] = c;
    }
    F::template fft<false, false>(v, line, p, tws);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R1; ++r) line[F::sw(p + P * r)] = v[r];
    __syncthreads();
    if (!valid) return;
    OT* dst = reinterpret_cast<OT*>(a.out) + comp * a.out_cstr + (int64_t)i1 * a.out_s1 + (int64_t)i2 * a.out_s2;
    // e^{-i pi / (4n)} of the type-IV kinds
    double ps, pc;
    sincospi(-0.25 / (double)n, &ps, &pc);
    const C ph4 = mkc((T)pc, (T)ps);
    const bool first = a.postpro & PP_NULL_FIRST, last = a.postpro & PP_NULL_LAST, period = a.postpro & PP_ENFORCE_PERIOD;
    auto value = [&](int k) -> T {
        if (k >= n) return (k < nsrc) ? (T)src[k] : z;  // beyond the transform: the padded input stays
        switch (kind) {
            case LK_DCT1: return line[F::sw(k)].x;
            case LK_DST1: return -line[F::sw(k + 1)].y;
            case LK_DCT2: return cmul(tw[k], line[F::sw(k)]).x;
            case LK_DST2: return -cmul(tw[k + 1], line[F::sw(k + 1)]).y;
            case LK_DCT3: return line[F::sw(k)].x;
            case LK_DST3: return -line[F::sw(k)].y;
            case LK_DCT4: return (T)2 * cmul(ph4, cmul(tw[k], line[F::sw(k)])).x;
            default: return -(T)2 * cmul(ph4, cmul(tw[k], line[F::sw(k)])).y;
        }
    };
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int i = p + P * r;
        if (i >= a.nstore) continue;
        T y;
        if (first && i == 0) y = z;
        else if (last && i == a.ilast) y = z;
        else if (period && !first && !last && i == a.nfftw) y = value(0);
        else y = value(i);
        dst[i] = (OT)y;
    }
}

// ---------------------------------------------------------------- rows: r2r, half length
// DCT / DST II-IV of an even length n through one n/2-point complex register
// DFT (LH = n/2) instead of the n- or 2n-point DFT of the extended row:
//   II  (FAM 2): Makhoul's reordering v = (x_0, x_2, ..., x_3, x_1), the real
//                n-point DFT V of v by the packed LH-point DFT and the split,
//                Y_k = 2 Re(W_4n^k V_k), Y_{n-k} = -2 Im(W_4n^k V_k);
//   III (FAM 3): the inverse: V_k = W_4n^{-k} (x_k - i x_{n-k}) (Hermitian),
//                v = the real inverse DFT of V by the c2r pre-process and an
//                LH-point inverse DFT, y_{2m} = v_m, y_{2m+1} = v_{n-1-m};
//   IV  (FAM 4): t_j = (x_{2j} + i x_{n-1-2j}) W_8n^{4j+1}, T = DFT_LH(t),
//                Y_{2k} = 2 Re(T_k W_4n^{2k}), Y_{n-1-2k} = -2 Im(T_k W_4n^{2k}).
// The DST kinds reduce to the DCT ones: DST-II(x)_k = DCT-II((-1)^j x_j)_{n-1-k},
// DST-III(x)_k = (-1)^k DCT-III(x_{n-1-j})_k, DST-IV(x)_k = (-1)^k DCT-IV(x_{n-1-j})_k.
// The row is read with unit-stride loads (any alignment) and scattered to its
// packed place in shared memory; the outputs are gathered back in row order, so
// loads and stores are coalesced.  Outputs past n pass the input through and
// the post-processing of the row (null first / last, period copy) is applied
// as in row_r2r_kernel.  tw: W_n^q (q < n); tw2: W_4n^q; tws: the LH-point table.
// W_4n^q entries a half-length DCT family uses (q <= LH; IV: q < n), staged in
// shared memory when they take at most 8 KB
template <typename T, int FAM, int LH>
struct DctW4 {
    static constexpr int USED = (FAM == 4) ? 2 * LH : (FAM == 1 ? 0 : LH + 1);
    static constexpr bool SM = USED > 0 && USED * (int)sizeof(typename CT<T>::C) <= 8192;
    static constexpr int N = SM ? USED : 0;
};

// CTAs per SM the DCT rows ask the compiler for: four for FP32 lines of a
// first radix up to 16 (64 registers), else the column passes' figure;
// FLB_DCT_MINB / FLB_DCT_MINB_F64 > 0 override it for FP32 / FP64
#ifndef FLB_DCT_MINB
#define FLB_DCT_MINB 0
#endif
#ifndef FLB_DCT_MINB_F64
#define FLB_DCT_MINB_F64 0
#endif
template <typename T, int R1, int THREADS>
struct DctOcc {
    static constexpr int over = sizeof(T) == 8 ? FLB_DCT_MINB_F64 : FLB_DCT_MINB;
    static constexpr int dflt = (sizeof(T) == 4 && R1 <= 16 && THREADS == 256) ? 4 : Occ<THREADS>::blocks;
    static constexpr int blocks = over > 0 ? over : dflt;
};

// rows whose outputs need no per-element test store them from a compile-time
// unrolled loop (0: every output through the general test; 513 x 257 x 257
// node grid: DCT-III rows 140 -> 115 us, DCT-II rows 116 -> 107 us)
#ifndef FLB_DCT_PLAIN_STORE
#define FLB_DCT_PLAIN_STORE 1
#endif
// DCT-III rows of all N inputs pre-processed from registers and lane
// shuffles (0: from a staged copy of the row in shared memory; the same grid:
// 115 -> 112 us)
#ifndef FLB_DCT3_SHFL
#define FLB_DCT3_SHFL 1
#endif
// line stride of the DCT rows (complex elements): FP32 rows of 16 lanes share
// a warp two by two, and at F::SC (a multiple of 16) the second row's 4-byte
// accesses (the packed scatter, the output gather) hit the first row's banks;
// FLB_DCT_SC_PAD complex elements more put them 8 banks apart
#ifndef FLB_DCT_SC_PAD
#define FLB_DCT_SC_PAD 4
#endif
template <typename F, typename T>
struct DctSC {
    static constexpr int V = F::SC + ((sizeof(T) == 4 && F::P == 16) ? FLB_DCT_SC_PAD : 0);
};

template <typename T, typename IT, typename OT, int LH, int R1, int TR, int FAM>
__global__ void __launch_bounds__(TR * (LH / R1), DctOcc<T, R1, TR * (LH / R1)>::blocks) row_dct_kernel(const RowArgs a) {
    using F = RegFFT<T, LH, R1, true>;
    using C = typename CT<T>::C;
    constexpr int P = F::P, N = 2 * LH;
    constexpr bool WSM = FAM != 4 && RowTw<T, LH>::SM;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int p = threadIdx.x % P, rr = threadIdx.x / P;
    const int row = blockIdx.x * TR + rr;
    const int comp = blockIdx.y;
    const bool valid = row < a.nrows;
    const int i1 = valid ? row % a.n1 : 0, i2 = valid ? row / a.n1 : 0;
    // src0: the row; src: the transform's first input (fi into the row)
    const IT* src0 = reinterpret_cast<const IT*>(a.in) + comp * a.in_cstr + (int64_t)i1 * a.in_s1 + (int64_t)i2 * a.in_s2;
    const IT* src = src0 + a.fi;
    constexpr int SCD = DctSC<F, T>::V;
    C* line = sm + rr * SCD;
    T* lr = reinterpret_cast<T*>(line);
    const C* tws = stage_twiddles<F>(a.tws, sm + TR * SCD);
    C* wsm = sm + TR * SCD + F::TW_SMEM;
    if constexpr (WSM) stage_table_part<C, LH>(a.tw, wsm);
    // the W_4n^q of this family, staged while the row loads are in flight
    const C* w4 = reinterpret_cast<const C*>(a.tw2);
    if constexpr (DctW4<T, FAM, LH>::SM) {
        C* w4s = wsm + (WSM ? LH : 0);
        for (int e = threadIdx.x; e < DctW4<T, FAM, LH>::N; e += blockDim.x) cp_async<sizeof(C)>(w4s + e, w4 + e);
        w4 = w4s;
    }
    cp_async_commit();
    const bool dst = (a.kind == LK_DST1 || a.kind == LK_DST2 || a.kind == LK_DST3 || a.kind == LK_DST4);
    // DCT-III rows of all N inputs: pre-processed from registers and lane
    // shuffles instead of a staged copy of the row
    constexpr bool SHFL3 = FAM == 3 && FLB_DCT3_SHFL && P <= 32 && (P & (P - 1)) == 0;
    T u3[SHFL3 ? 2 * R1 : 1];
    // inputs the transform reads: n (DCT-I n = LH + 1, DST-I n = LH - 1), else up to N
    const int ntr = (FAM == 1) ? a.n : N;
    const int nld = valid ? (a.nin - a.fi < ntr ? a.nin - a.fi : ntr) : 0;
    const T z = (T)0;
    // real m of the packed line: z_j = (r_{2j}, r_{2j+1}) at line[sw(j)]
    auto slot = [](int m) { return 2 * F::sw(m >> 1) + (m & 1); };
    auto stage = [&](auto full) {
#pragma unroll
        for (int r = 0; r < 2 * R1; ++r) {
            const int i = p + P * r;
            const T u = (decltype(full)::value || i < nld) ? (T)src[i] : z;
            if constexpr (FAM == 3 && 64 % P == 0) {
                // slot(i) = i + 2 (i >> 6), and (p + P r) >> 6 = (P r) >> 6 for p < P | 64
                lr[p + (P * r + 2 * ((P * r) >> 6))] = u;
            } else if constexpr (FAM == 2 && P % 2 == 0 && 128 % P == 0) {
                // i = p + P r has the parity of p: even i -> m = q + (P/2) r, odd i ->
                // m = N - 1 - (P/2) r - q (q = p >> 1); slot(m) = m + 2 (m >> 6), where q
                // never carries across a multiple of 64
                constexpr int H = P / 2;
                const int q = p >> 1;
                if (p & 1) {
                    const int M = N - 1 - H * r;
                    lr[(M + 2 * (M >> 6)) - q] = dst ? -u : u;
                } else {
                    lr[q + (H * r + 2 * ((H * r) >> 6))] = u;
                }
            } else {
                int m;
                if constexpr (FAM == 2) {
                    m = (i & 1) ? N - 1 - (i >> 1) : (i >> 1);
                } else if constexpr (FAM == 3) {
                    m = i;
                } else {
                    const int ii = dst ? N - 1 - i : i;
                    m = (ii & 1) ? N - ii : ii;  // x_{2j} -> r_{2j}; x_{n-1-2j} -> r_{2j+1}
                }
                lr[slot(m)] = (FAM == 2 && dst && (i & 1)) ? -u : u;
            }
        }
    };
    if constexpr (FAM == 1) {
        // the 2 LH-point real extension z of the row, packed: DCT-I z_j = x_j for
        // j <= LH, z_{2LH-j} = x_j; DST-I z_{j+1} = x_j, z_{2LH-1-j} = -x_j,
        // z_0 = z_LH = 0.  Lane p loads x_i, i = p + P r (i < LH), lane 0 also
        // i = LH; every x_i lands in its one or two places.
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int i = p + P * r;
            const T u = (i < nld) ? (T)src[i] : z;
            if (dst) {
                lr[slot(i + 1)] = u;
                lr[slot(N - 1 - i)] = -u;
            } else {
                lr[slot(i)] = u;
                if (i > 0) lr[slot(N - i)] = u;
            }
        }
        if (p == 0) {
            const T u = (!dst && LH < nld) ? (T)src[LH] : z;
            lr[slot(LH)] = u;  // DCT-I: x_LH; DST-I: z_LH = 0
            if (dst) lr[slot(0)] = z;
        }
    } else if (SHFL3 && !dst && nld >= N) {
        // DCT-III rows held in registers: u[r] = x_{p + P r}
#pragma unroll
        for (int r = 0; r < 2 * R1; ++r) u3[r] = (T)src[p + P * r];
    } else {
        // rows that hold all N inputs load them without a test per element
        if (nld >= N) stage(std::true_type{});
        else stage(std::false_type{});
    }
    cp_async_wait<0>();
    __syncthreads();
    const C* wn = WSM ? wsm : reinterpret_cast<const C*>(a.tw);
    C v[R1];
    if constexpr (FAM == 1 || FAM == 2) {
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = line[F::sw(p + P * r)];
    } else if constexpr (FAM == 4) {
        double ps, pc;
        sincospi(-0.25 / (double)N, &ps, &pc);
        const C w8 = mkc((T)pc, (T)ps);
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int j = p + P * r;
            v[r] = cmul(cmul(line[F::sw(j)], w4[2 * j]), w8);
        }
    } else if (SHFL3 && !dst && nld >= N) {
        // x_k = u[r] and x_{LH+k} = u[r + R1] are this lane's (k = p + P r); for
        // p > 0, x_{N-k} and x_{LH-k} are lane P - p's u[2 R1 - 1 - r] and
        // u[R1 - 1 - r]; lane 0 holds its own (x_N = 0)
        const int lane = threadIdx.x & 31;
        const unsigned gm = (P >= 32) ? 0xffffffffu : (((1u << (P & 31)) - 1u) << (lane & ~(P - 1)));
        const int src_lane = (P - p) & (P - 1);
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = p + P * r;
            const T sn = __shfl_sync(gm, u3[2 * R1 - 1 - r], src_lane, P);
            const T sl = __shfl_sync(gm, u3[R1 - 1 - r], src_lane, P);
            const T xn = (p == 0) ? (r == 0 ? z : u3[(2 * R1 - r) % (2 * R1)]) : sn;
            const T xl = (p == 0) ? u3[R1 - r] : sl;
            C xk = cmulc(mkc(u3[r], -xn), w4[k]);
            C xm = cmulc(mkc(xl, -u3[r + R1]), w4[LH - k]);
            if (k == 0) {
                xk.y = z;
                xm.y = z;
            }
            xm = cconj(xm);
            const C A = cadd(xk, xm);
            const C B = cmul(csub(xk, xm), cconj(wn[k]));
            v[r] = mkc(A.x - B.y, A.y + B.x);
        }
    } else {
        auto x = [&](int i) { return (i >= 0 && i < N) ? lr[slot(i)] : z; };
        auto V = [&](int q) {
            const T xa = dst ? x(N - 1 - q) : x(q), xb = dst ? x(q - 1) : x(N - q);
            return cmulc(mkc(xa, -xb), w4[q]);  // W_4n^{-q} (xa - i xb)
        };
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = p + P * r;
            C xk = V(k), xm = V(LH - k);
            if (k == 0) {
                xk.y = z;
                xm.y = z;
            }
            xm = cconj(xm);
            const C A = cadd(xk, xm);
            const C B = cmul(csub(xk, xm), cconj(wn[k]));
            v[r] = mkc(A.x - B.y, A.y + B.x);
        }
    }
    F::template fft<false, FAM == 3>(v, line, p, tws);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R1; ++r) line[F::sw(p + P * r)] = v[r];
    if constexpr (FAM == 2) {
        // (Y_k, Y_{n-k}) at line[sw(k)], k < LH; (Y_0, Y_LH) at k = 0
        __syncthreads();
        constexpr T RT2 = (T)1.4142135623730950488;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = p + P * r;
            const C zk = v[r];
            const C zm = cconj(line[F::sw(k == 0 ? 0 : LH - k)]);
            const C e = cadd(zk, zm);
            const C w = cmul(wn[k], csub(zk, zm));
            const C Pk = cmul(w4[k], mkc((T)0.5 * (e.x + w.y), (T)0.5 * (e.y - w.x)));
            v[r] = mkc((T)2 * Pk.x, (T)-2 * Pk.y);
            if (r == 0 && p == 0) v[0].y = RT2 * (zk.x - zk.y);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R1; ++r) line[F::sw(p + P * r)] = v[r];
    } else if constexpr (FAM == 4) {
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = p + P * r;
            const C u = cmul(v[r], w4[2 * k]);
            line[F::sw(k)] = mkc((T)2 * u.x, (T)-2 * u.y);  // (Y_{2k}, Y_{n-1-2k})
        }
    } else if constexpr (FAM == 1) {
        // the N-point real DFT Z of z from the packed LH-point DFT C:
        // Z_k = E_k + W_N^k O_k, E_k = (C_k + conj C_{LH-k}) / 2,
        // O_k = (C_k - conj C_{LH-k}) / 2i (C_LH = C_0); DCT-I Y_k = Re Z_k
        // (k <= LH, Z_LH = Re C_0 - Im C_0), DST-I Y_{k-1} = -Im Z_k (0 < k < LH).
        // The real outputs are then laid out in row order over the line.
        __syncthreads();
        T y[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = p + P * r;
            const C zk = v[r];
            const C zm = cconj(line[F::sw(k == 0 ? 0 : LH - k)]);
            const C e = cadd(zk, zm);
            const C w = cmul(wn[k], csub(zk, zm));
            y[r] = dst ? (T)-0.5 * (e.y - w.x) : (T)0.5 * (e.x + w.y);
        }
        const T ylh = v[0].x - v[0].y;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = p + P * r;
            if (!dst) lr[k] = y[r];
            else if (k > 0) lr[k - 1] = y[r];
        }
        if (p == 0 && !dst) lr[LH] = ylh;
    }
    __syncthreads();
    if (!valid) return;
    OT* out = reinterpret_cast<OT*>(a.out) + comp * a.out_cstr + (int64_t)i1 * a.out_s1 + (int64_t)i2 * a.out_s2;
    auto value = [&](int i) -> T {
        if constexpr (FAM == 2) {
            const int k = dst ? N - 1 - i : i;
            return k < LH ? line[F::sw(k)].x : (k == LH ? line[0].y : line[F::sw(N - k)].y);
        } else if constexpr (FAM == 3) {
            const T y = lr[slot((i & 1) ? N - 1 - (i >> 1) : (i >> 1))];
            return (dst && (i & 1)) ? -y : y;
        } else if constexpr (FAM == 1) {
            return lr[i];
        } else {
            const T y = (i & 1) ? line[F::sw((N - 1 - i) >> 1)].y : line[F::sw(i >> 1)].x;
            return (dst && (i & 1)) ? -y : y;
        }
    };
    const bool first = a.postpro & PP_NULL_FIRST, last = a.postpro & PP_NULL_LAST, period = a.postpro & PP_ENFORCE_PERIOD;
    // row element i: transform output i - fo, else the row's input stays
    auto outv = [&](int i) -> T {
        const int k = i - a.fo;
        if (k < 0 || k >= ntr) return (i < a.nin) ? (T)src0[i] : z;
        return value(k);
    };
    auto store = [&](int i) {
        T y;
        if (first && i == 0) y = z;
        else if (last && i == a.ilast) y = z;
        else if (period && !first && !last && i == a.nfftw) y = outv(0);
        else y = outv(i);
        out[i] = (OT)y;
    };
    // the usual row: transform outputs from index 0, all N of them stored, no
    // period copy and no nulled output among them but (maybe) output 0
    const bool plain = FAM != 1 && FLB_DCT_PLAIN_STORE && a.fo == 0 && !period && a.nstore >= N && (!last || a.ilast >= N);
    if (plain) {
        // outputs i < N as p + P r (compile-time r), then the rest
#pragma unroll
        for (int r = 0; r < 2 * R1; ++r) {
            const int i = p + P * r;
            T y = value(i);
            if (r == 0 && first && p == 0) y = z;
            out[i] = (OT)y;
        }
        for (int i = N + p; i < a.nstore; i += P) store(i);
    } else if constexpr (FAM == 3) {
#pragma unroll
        for (int r = 0; r < 2 * R1; ++r) {
            const int i = p + P * r;
            if (i < a.nstore) store(i);
        }
        for (int i = N + p; i < a.nstore; i += P) store(i);
    } else {
        for (int i = p; i < a.nstore; i += P) store(i);
    }
}

// ---------------------------------------------------------------- rows: c2r
// OT: type of the real output; HALF: nout = Lh (the row is truncated to half)
template <typename T, typename OT, int LH, int R1, int TR, bool HALF>
__global__ void __launch_bounds__(TR * (LH / R1), (Occ<TR * (LH / R1), false, RowTiles<T, LH, R1>::WIDE, Row3<T, R1>::ON>::blocks)) row_c2r_kernel(const __grid_constant__ RowArgs a) {
    using F = RegFFT<T, LH, R1, true, Row3<T, R1>::ON>;
    using C = typename CT<T>::C;
    using V = typename Vec2<OT>::V;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int p = threadIdx.x % F::P, rr = threadIdx.x / F::P;
    const int row = blockIdx.x * TR + rr;
    const int comp = blockIdx.y;
    const bool valid = row < a.nrows;
    const int i1 = valid ? row % a.n1 : 0, i2 = valid ? row / a.n1 : 0;
    prefetch_ahead<true>(a.pf, TR, a.n1);
    C* line = sm + rr * F::SC;
    const C* tws = stage_twiddles<F>(a.tws, sm + TR * F::SC);
    C* wsm = sm + TR * F::SC + F::TW_SMEM;
    if constexpr (RowTw<T, LH>::SM) {
        stage_table_part<C, LH>(a.tw, wsm);
        cp_async_commit();
    }
    const C* src = reinterpret_cast<const C*>(a.in) + comp * a.in_cstr + (int64_t)i1 * a.in_s1 + (int64_t)i2 * a.in_s2;
    // stage the half spectrum X[0..LH] (line positions 0..LH-1, X[LH] kept aside in registers);
    // rows past the end read the array's first element and drop it (no branch)
    const C* srcv = valid ? src : reinterpret_cast<const C*>(a.in);
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int k = p + F::P * r;
        const C t = srcv[valid ? k : 0];
        line[F::sw(k)] = valid ? t : mkc((T)0, (T)0);
    }
    const C xl = srcv[valid ? LH : 0];
    const C xlh = valid ? xl : mkc((T)0, (T)0);
    if constexpr (F::TWS || RowTw<T, LH>::SM) cp_async_wait<0>();
    __syncthreads();
    // Z'_k = A_k + i B_k, A = X_k + conj X_{LH-k}, B = (X_k - conj X_{LH-k}) W_L^{-k};
    // Im X_0 and Im X_LH do not enter a real inverse transform
    const C* tw = (RowTw<T, LH>::SM ? wsm : reinterpret_cast<const C*>(a.tw)) + p;
    C v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int k = p + F::P * r;
        C xk = line[F::sw(k)];
        C xm = line[F::sw(k == 0 ? 0 : LH - k)];
        if (k == 0) {
            xm = xlh;
            xk.y = (T)0;
            xm.y = (T)0;
        }
        xm = cconj(xm);
        const C A = cadd(xk, xm);
        const C B = cmul(csub(xk, xm), cconj(tw[F::P * r]));
        v[r] = mkc(A.x - B.y, A.y + B.x);
    }
    F::template fft<false, true>(v, line, p, tws);
    if (valid) {
        OT* dst = reinterpret_cast<OT*>(a.out) + comp * a.out_cstr + (int64_t)i1 * a.out_s1 + (int64_t)i2 * a.out_s2 + 2 * p;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int j = p + F::P * r;
            if (HALF) {
                if (r < R1 / 2) *reinterpret_cast<V*>(dst + 2 * F::P * r) = V{(OT)v[r].x, (OT)v[r].y};
            } else {
                if (2 * j + 1 < a.nout) *reinterpret_cast<V*>(dst + 2 * F::P * r) = V{(OT)v[r].x, (OT)v[r].y};
                else if (2 * j < a.nout) dst[2 * F::P * r] = (OT)v[r].x;
            }
        }
    }
}

// ---------------------------------------------------------------- launchers

// per-unit launchers (instantiated in fast_col_*.cu / fast_row.cu)
cudaError_t launch_col_f32_m01(int mode, int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_col_f32_m2(int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_col_f64_m01(int mode, int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_col_f64_m2(int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_col_f32_m3(int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_rowfused_f32(int rot, int sh, int L, const RowFusedArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_rowfused_f64(int rot, int sh, int L, const RowFusedArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_col_f64_m3(int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_row_units(int f64, int c2r, int xt64, bool half, int L, const RowArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_colreal_f32(int c2r, int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s);
// FP32 columns whose real side is the user's doubles
cudaError_t launch_colreal_f32u(int c2r, int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_r2r_units(int f64, int in64, int out64, int M, const RowArgs& a, int ncomp, cudaStream_t s);
// n: the real DFT length of the extension (M)
cudaError_t launch_dct1_units(int f64, int in64, int out64, int n, const RowArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_dct2_units(int f64, int in64, int out64, int n, const RowArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_dct3_units(int f64, int in64, int out64, int n, const RowArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_dct4_units(int f64, int in64, int out64, int n, const RowArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_colreal_f64(int c2r, int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s);

template <typename T, int L, int R1, int TX, int MODE, int SH>
inline cudaError_t launch_col_t(const ColArgs& a, int ncomp, cudaStream_t s) {
    using F = RegFFT<T, L, R1, false, Fwd3<T, MODE, R1>::ON && TX * (L / R1) == 256>;
    const size_t smem = (size_t)(TX * F::SC + F::TW_SMEM) * sizeof(typename CT<T>::C) +
                        (MODE == 2 ? (size_t)GStage<L>::N * TX * sizeof(T) : 0);
    static std::atomic<unsigned long long> attr{0};
    if (cudaError_t e = smem_attr_once(attr, col_dft_kernel<T, L, R1, TX, MODE, SH>, smem); e != cudaSuccess) return e;
    dim3 grid((a.nx + TX - 1) / TX, a.nouter, ncomp);
    col_dft_kernel<T, L, R1, TX, MODE, SH><<<grid, TX * F::P, smem, s>>>(a);
    return cudaGetLastError();
}

// CTA tiles of a column pass: THREADS threads = TX columns x P threads per
// line.  Two tiles are compiled per length (256 and 128 threads); the default
// is 256 threads except at L = 512, where 128 threads (8 FP32 columns) won,
// and for the FP64 passes at 255 registers (first radix 32, or fused), which
// run two 128-thread CTAs per SM; the autotuner (Solver::autotune_passes) may
// pick the other per pass.
template <typename T, int L, int THREADS, int MODE, int SH>
inline cudaError_t launch_col_threads(const ColArgs& a, int ncomp, cudaStream_t s) {
    constexpr int R1 = fast_radix1_mode(L, sizeof(T) == 8, MODE);
    constexpr int TX = THREADS / (L / R1);
    static_assert(TX >= 1, "tile narrower than one column");
    return launch_col_t<T, L, R1, TX, MODE, SH>(a, ncomp, s);
}

// default: 128 threads at L = 512 and for the FP64 passes at 255 registers
// (two CTAs per SM), else 256
inline int col_tile_threads(int L, int tile, bool prefer128 = false) {
    if (tile == COL_TILE_256) return 256;
    if (tile == COL_TILE_128) return 128;
    return (L == 512 || prefer128) ? 128 : 256;
}

template <typename T, int MODE, int SH>
inline cudaError_t launch_col_mode(int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    const bool wide =
        col_tile_threads(L, a.tile, (sizeof(T) == 8 && (MODE == 2 || L % 3 != 0)) || fast_radix1_mode(L, sizeof(T) == 8, MODE) == 48) == 256;
    switch (L) {
        case 64: return wide ? launch_col_threads<T, 64, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 64, 128, MODE, SH>(a, ncomp, s);
        case 128: return wide ? launch_col_threads<T, 128, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 128, 128, MODE, SH>(a, ncomp, s);
        case 256: return wide ? launch_col_threads<T, 256, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 256, 128, MODE, SH>(a, ncomp, s);
        case 512: return wide ? launch_col_threads<T, 512, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 512, 128, MODE, SH>(a, ncomp, s);
        case 1024: return wide ? launch_col_threads<T, 1024, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 1024, 128, MODE, SH>(a, ncomp, s);
        case 2048: return wide ? launch_col_threads<T, 2048, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 2048, 128, MODE, SH>(a, ncomp, s);
        case 48: return wide ? launch_col_threads<T, 48, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 48, 128, MODE, SH>(a, ncomp, s);
        case 96: return wide ? launch_col_threads<T, 96, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 96, 128, MODE, SH>(a, ncomp, s);
        case 192: return wide ? launch_col_threads<T, 192, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 192, 128, MODE, SH>(a, ncomp, s);
        case 384: return wide ? launch_col_threads<T, 384, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 384, 128, MODE, SH>(a, ncomp, s);
        case 768: return wide ? launch_col_threads<T, 768, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 768, 128, MODE, SH>(a, ncomp, s);
        case 1536: return wide ? launch_col_threads<T, 1536, 256, MODE, SH>(a, ncomp, s) : launch_col_threads<T, 1536, 128, MODE, SH>(a, ncomp, s);
    }
    return cudaErrorInvalidValue;
}

// ROT fused pass: ncomp = 3 x (groups of three components)
template <typename T, int L, int SH>
inline cudaError_t launch_rot_t(const ColArgs& a, int ncomp, cudaStream_t s) {
    using RT = RotTile<T, L>;
    using F = RegFFT<T, L, RT::R1>;
    constexpr size_t smem =
        (size_t)(3 * RT::TX * F::SC + F::TW_SMEM) * sizeof(typename CT<T>::C) + (size_t)GStage<L>::N * RT::TX * sizeof(T);
    if constexpr (smem > 227 * 1024) {
        return cudaErrorInvalidValue;
    } else {
        if (ncomp % 3 != 0 || ncomp / 3 > 65535) return cudaErrorInvalidValue;
        static std::atomic<unsigned long long> attr{0};
        if (cudaError_t e = smem_attr_once(attr, col_rot_kernel<T, L, RT::R1, RT::TX, SH>, smem); e != cudaSuccess) return e;
        dim3 grid((a.nx + RT::TX - 1) / RT::TX, a.nouter, ncomp / 3);
        col_rot_kernel<T, L, RT::R1, RT::TX, SH><<<grid, RT::THREADS, smem, s>>>(a);
        return cudaGetLastError();
    }
}

template <typename T, int SH>
inline cudaError_t launch_rot_len(int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    switch (L) {
        case 48: return launch_rot_t<T, 48, SH>(a, ncomp, s);
        case 64: return launch_rot_t<T, 64, SH>(a, ncomp, s);
        case 96: return launch_rot_t<T, 96, SH>(a, ncomp, s);
        case 128: return launch_rot_t<T, 128, SH>(a, ncomp, s);
        case 192: return launch_rot_t<T, 192, SH>(a, ncomp, s);
        case 256: return launch_rot_t<T, 256, SH>(a, ncomp, s);
        case 384: return launch_rot_t<T, 384, SH>(a, ncomp, s);
        case 512: return launch_rot_t<T, 512, SH>(a, ncomp, s);
        case 768: return launch_rot_t<T, 768, SH>(a, ncomp, s);
        case 1024: return launch_rot_t<T, 1024, SH>(a, ncomp, s);
        case 1536: return launch_rot_t<T, 1536, SH>(a, ncomp, s);
        case 2048: return launch_rot_t<T, 2048, SH>(a, ncomp, s);
    }
    return cudaErrorInvalidValue;
}

template <typename T>
inline cudaError_t launch_rot_shape(int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    if (sh == SH_FULL) return launch_rot_len<T, SH_FULL>(L, a, ncomp, s);
    if (sh == SH_HALF) return launch_rot_len<T, SH_HALF>(L, a, ncomp, s);
    return launch_rot_len<T, SH_ANY>(L, a, ncomp, s);
}

template <typename T, typename RT, int L, bool C2R, int SH>
inline cudaError_t launch_colreal_t(const ColArgs& a, int ncomp, cudaStream_t s) {
    constexpr int R1 = fast_radix1_colreal(L, sizeof(T) == 8);
    constexpr int TX = (L == 512 ? 128 : 256) / (L / R1);
    static_assert(TX >= 1, "tile narrower than one column");
    using F = RegFFT<T, L, R1>;
    if (a.pairs) {
        // column pairs: the same threads per CTA, each line two columns
        constexpr int TXP = TX;
        const size_t smem = (size_t)(TXP * F::SC + F::TW_SMEM) * sizeof(typename CT<T>::C);
        static std::atomic<unsigned long long> attr{0};
        if (cudaError_t e = smem_attr_once(attr, col_real_pair_kernel<T, RT, L, R1, TXP, C2R, SH>, smem); e != cudaSuccess) return e;
        dim3 grid(((a.nx + 1) / 2 + TXP - 1) / TXP, a.nouter, ncomp);
        col_real_pair_kernel<T, RT, L, R1, TXP, C2R, SH><<<grid, TXP * F::P, smem, s>>>(a);
        return cudaGetLastError();
    }
    const size_t smem = (size_t)(TX * F::SC + F::TW_SMEM) * sizeof(typename CT<T>::C);
    static std::atomic<unsigned long long> attr{0};
    if (cudaError_t e = smem_attr_once(attr, col_real_kernel<T, RT, L, R1, TX, C2R, SH>, smem); e != cudaSuccess) return e;
    dim3 grid((a.nx + TX - 1) / TX, a.nouter, ncomp);
    col_real_kernel<T, RT, L, R1, TX, C2R, SH><<<grid, TX * F::P, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename T, typename RT, bool C2R, int SH>
inline cudaError_t launch_colreal_len(int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    switch (L) {
        case 48: return launch_colreal_t<T, RT, 48, C2R, SH>(a, ncomp, s);
        case 64: return launch_colreal_t<T, RT, 64, C2R, SH>(a, ncomp, s);
        case 96: return launch_colreal_t<T, RT, 96, C2R, SH>(a, ncomp, s);
        case 128: return launch_colreal_t<T, RT, 128, C2R, SH>(a, ncomp, s);
        case 192: return launch_colreal_t<T, RT, 192, C2R, SH>(a, ncomp, s);
        case 256: return launch_colreal_t<T, RT, 256, C2R, SH>(a, ncomp, s);
        case 384: return launch_colreal_t<T, RT, 384, C2R, SH>(a, ncomp, s);
        case 512: return launch_colreal_t<T, RT, 512, C2R, SH>(a, ncomp, s);
        case 768: return launch_colreal_t<T, RT, 768, C2R, SH>(a, ncomp, s);
        case 1024: return launch_colreal_t<T, RT, 1024, C2R, SH>(a, ncomp, s);
        case 1536: return launch_colreal_t<T, RT, 1536, C2R, SH>(a, ncomp, s);
        case 2048: return launch_colreal_t<T, RT, 2048, C2R, SH>(a, ncomp, s);
    }
    return cudaErrorInvalidValue;
}

template <typename T, typename RT, bool C2R>
inline cudaError_t launch_colreal_shape(int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    if (sh == SH_FULL) return launch_colreal_len<T, RT, C2R, SH_FULL>(L, a, ncomp, s);
    if (sh == SH_HALF) return launch_colreal_len<T, RT, C2R, SH_HALF>(L, a, ncomp, s);
    return launch_colreal_len<T, RT, C2R, SH_ANY>(L, a, ncomp, s);
}

template <typename T, int MODE>
inline cudaError_t launch_col_shape(int sh, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    if (sh == SH_FULL) return launch_col_mode<T, MODE, SH_FULL>(L, a, ncomp, s);
    if (sh == SH_HALF) return launch_col_mode<T, MODE, SH_HALF>(L, a, ncomp, s);
    if constexpr (MODE == 2)
        if (sh == SH_HALF1) return launch_col_mode<T, MODE, SH_HALF1>(L, a, ncomp, s);
    return launch_col_mode<T, MODE, SH_ANY>(L, a, ncomp, s);
}

template <typename T, typename IT, typename OT, int M>
inline cudaError_t launch_r2r_t(const RowArgs& a, int ncomp, cudaStream_t s) {
    constexpr int R1 = fast_radix1_of(M, sizeof(T) == 8);
    using F = RegFFT<T, M, R1, true>;
    constexpr int TR = (F::P >= 256) ? 1 : 256 / F::P;
    const size_t smem = (size_t)(TR * F::SC + F::TW_SMEM) * sizeof(typename CT<T>::C);
    static std::atomic<unsigned long long> attr{0};
    if (cudaError_t e = smem_attr_once(attr, row_r2r_kernel<T, IT, OT, M, R1, TR>, smem); e != cudaSuccess) return e;
    dim3 grid((a.nrows + TR - 1) / TR, ncomp);
    row_r2r_kernel<T, IT, OT, M, R1, TR><<<grid, TR * F::P, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename T, typename IT, typename OT>
inline cudaError_t launch_r2r_len(int M, const RowArgs& a, int ncomp, cudaStream_t s) {
    switch (M) {
        case 64: return launch_r2r_t<T, IT, OT, 64>(a, ncomp, s);
        case 96: return launch_r2r_t<T, IT, OT, 96>(a, ncomp, s);
        case 128: return launch_r2r_t<T, IT, OT, 128>(a, ncomp, s);
        case 192: return launch_r2r_t<T, IT, OT, 192>(a, ncomp, s);
        case 256: return launch_r2r_t<T, IT, OT, 256>(a, ncomp, s);
        case 384: return launch_r2r_t<T, IT, OT, 384>(a, ncomp, s);
        case 512: return launch_r2r_t<T, IT, OT, 512>(a, ncomp, s);
        case 768: return launch_r2r_t<T, IT, OT, 768>(a, ncomp, s);
        case 1024: return launch_r2r_t<T, IT, OT, 1024>(a, ncomp, s);
        case 2048: return launch_r2r_t<T, IT, OT, 2048>(a, ncomp, s);
    }
    return cudaErrorInvalidValue;
}

template <typename T, typename IT, typename OT, int LH, int FAM>
inline cudaError_t launch_dct_t(const RowArgs& a, int ncomp, cudaStream_t s) {
    constexpr int R1 = fast_radix1_dct(LH, sizeof(T) == 8);
    using F = RegFFT<T, LH, R1, true>;
    constexpr int TR = (F::P >= 256) ? 1 : 256 / F::P;
    const size_t smem =
        (size_t)(TR * DctSC<F, T>::V + F::TW_SMEM + (FAM != 4 ? RowTw<T, LH>::N : 0) + DctW4<T, FAM, LH>::N) * sizeof(typename CT<T>::C);
    static std::atomic<unsigned long long> attr{0};
    if (cudaError_t e = smem_attr_once(attr, row_dct_kernel<T, IT, OT, LH, R1, TR, FAM>, smem); e != cudaSuccess) return e;
    dim3 grid((a.nrows + TR - 1) / TR, ncomp);
    row_dct_kernel<T, IT, OT, LH, R1, TR, FAM><<<grid, TR * F::P, smem, s>>>(a);
    return cudaGetLastError();
}

// n: the (even) transform length; LH = n / 2
template <typename T, typename IT, typename OT, int FAM>
inline cudaError_t launch_dct_len(int n, const RowArgs& a, int ncomp, cudaStream_t s) {
    switch (n) {
        case 64: return launch_dct_t<T, IT, OT, 32, FAM>(a, ncomp, s);
        case 96: return launch_dct_t<T, IT, OT, 48, FAM>(a, ncomp, s);
        case 128: return launch_dct_t<T, IT, OT, 64, FAM>(a, ncomp, s);
        case 192: return launch_dct_t<T, IT, OT, 96, FAM>(a, ncomp, s);
        case 256: return launch_dct_t<T, IT, OT, 128, FAM>(a, ncomp, s);
        case 384: return launch_dct_t<T, IT, OT, 192, FAM>(a, ncomp, s);
        case 512: return launch_dct_t<T, IT, OT, 256, FAM>(a, ncomp, s);
        case 768: return launch_dct_t<T, IT, OT, 384, FAM>(a, ncomp, s);
        case 1024: return launch_dct_t<T, IT, OT, 512, FAM>(a, ncomp, s);
        case 1536: return launch_dct_t<T, IT, OT, 768, FAM>(a, ncomp, s);
        case 2048: return launch_dct_t<T, IT, OT, 1024, FAM>(a, ncomp, s);
    }
    return cudaErrorInvalidValue;
}

template <int FAM>
inline cudaError_t launch_dct_types(int f64, int in64, int out64, int n, const RowArgs& a, int ncomp, cudaStream_t s) {
    if (f64) return launch_dct_len<double, double, double, FAM>(n, a, ncomp, s);
    if (in64 && !out64) return launch_dct_len<float, double, float, FAM>(n, a, ncomp, s);
    if (!in64 && out64) return launch_dct_len<float, float, double, FAM>(n, a, ncomp, s);
    if (!in64 && !out64) return launch_dct_len<float, float, float, FAM>(n, a, ncomp, s);
    return cudaErrorInvalidValue;
}

template <typename T, typename XT, int LH, int R1, bool C2R, bool HALF>
inline cudaError_t launch_row_t(const RowArgs& a, int ncomp, cudaStream_t s) {
    using F = RegFFT<T, LH, R1, true, Row3<T, R1>::ON>;
    constexpr int TR = RowTiles<T, LH, R1>::TR;
    const size_t smem = (size_t)(TR * F::SC + F::TW_SMEM + RowTw<T, LH>::N) * sizeof(typename CT<T>::C);
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e;
    if constexpr (C2R) e = smem_attr_once(attr, row_c2r_kernel<T, XT, LH, R1, TR, HALF>, smem);
    else e = smem_attr_once(attr, row_r2c_kernel<T, XT, LH, R1, TR, HALF>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((a.nrows + TR - 1) / TR, ncomp);
    if constexpr (C2R) row_c2r_kernel<T, XT, LH, R1, TR, HALF><<<grid, TR * F::P, smem, s>>>(a);
    else row_r2c_kernel<T, XT, LH, R1, TR, HALF><<<grid, TR * F::P, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename T, typename XT, bool C2R, bool HALF>
inline cudaError_t launch_row_len(int L, const RowArgs& a, int ncomp, cudaStream_t s) {
    constexpr bool F64 = sizeof(T) == 8;
    switch (L) {
        case 128: return launch_row_t<T, XT, 64, fast_radix1_row(64, F64), C2R, HALF>(a, ncomp, s);
        case 256: return launch_row_t<T, XT, 128, fast_radix1_row(128, F64), C2R, HALF>(a, ncomp, s);
        case 512: return launch_row_t<T, XT, 256, fast_radix1_row(256, F64), C2R, HALF>(a, ncomp, s);
        case 1024: return launch_row_t<T, XT, 512, fast_radix1_row(512, F64), C2R, HALF>(a, ncomp, s);
        case 2048: return launch_row_t<T, XT, 1024, fast_radix1_row(1024, F64), C2R, HALF>(a, ncomp, s);
        case 4096: return launch_row_t<T, XT, 2048, fast_radix1_row(2048, F64), C2R, HALF>(a, ncomp, s);
        case 48: return launch_row_t<T, XT, 24, fast_radix1_row(24, F64), C2R, HALF>(a, ncomp, s);
        case 64: return launch_row_t<T, XT, 32, fast_radix1_row(32, F64), C2R, HALF>(a, ncomp, s);
        case 96: return launch_row_t<T, XT, 48, fast_radix1_row(48, F64), C2R, HALF>(a, ncomp, s);
        case 192: return launch_row_t<T, XT, 96, fast_radix1_row(96, F64), C2R, HALF>(a, ncomp, s);
        case 384: return launch_row_t<T, XT, 192, fast_radix1_row(192, F64), C2R, HALF>(a, ncomp, s);
        case 768: return launch_row_t<T, XT, 384, fast_radix1_row(384, F64), C2R, HALF>(a, ncomp, s);
        case 1536: return launch_row_t<T, XT, 768, fast_radix1_row(768, F64), C2R, HALF>(a, ncomp, s);
        case 3072: return launch_row_t<T, XT, 1536, fast_radix1_row(1536, F64), C2R, HALF>(a, ncomp, s);
    }
    return cudaErrorInvalidValue;
}

template <typename T, typename XT, bool C2R>
inline cudaError_t launch_row_half(bool half, int L, const RowArgs& a, int ncomp, cudaStream_t s) {
    return half ? launch_row_len<T, XT, C2R, true>(L, a, ncomp, s) : launch_row_len<T, XT, C2R, false>(L, a, ncomp, s);
}

}  // namespace flb
