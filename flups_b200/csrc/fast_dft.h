// Arguments and launchers of the register-resident power-of-two DFT passes
// (fast_dft.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace flb {

// L2 prefetch of the block `dist` launches ahead: a tensor map over the
// pass's input (8-byte units, dims x, line / row, outer, component) and the
// number of boxes per block along dim 0 (rows) or dim 1 (columns); nbox = 0
// disables it.  The map is a member of the kernel's __grid_constant__
// argument, so the TMA unit reads it from parameter space.
struct Prefetch {
    CUtensorMap map;
    int nbox, dist, step;
};

struct ColArgs {
    const void* in;
    void* out;
    int nx;                 // columns along x (complex elements)
    int nin, nout;          // loaded / stored extent along the line (zero beyond nin)
    int64_t in_lstr, in_ostr, in_cstr;     // element strides: along line, outer, component
    int64_t out_lstr, out_ostr, out_cstr;
    int nouter;
    const void* tws;        // later-stage twiddle table of the L-point DFT (fast_stage_table)
    // fused multiply
    const void* green;
    int64_t g_x, g_line, g_outer;          // folded Green strides
    int f_x, f_line, f_outer;              // fold lengths (0 = none)
    double normfact;
    int tile;               // CTA tile: COL_TILE_DEFAULT, COL_TILE_256 or COL_TILE_128 threads
    int period;             // r2c / c2r columns: index that receives a copy of index 0, or -1
    int real64;             // r2c / c2r columns in FP32: the real side holds doubles (the user's array)
    int pairs;              // r2c / c2r columns two at a time (aligned pairs: even strides, 16-byte bases)
    Prefetch pf;            // column passes 0 / 1 along a short-stride axis
    // ROT fused pass (mode 3): the curl's wave-number symbols K_{d,c}(i), one
    // table of complex working-precision values per direction d and component
    // c at ksym + (3 d + c) kstr, indexed by the spectral index along d; the
    // directions of the line and of the outer index
    const void* ksym;
    int kstr;
    int ax_line, ax_outer;
    // z-slab solves: the column arrays of every rank (device or peer memory)
    // in place of `out` (mode 0) or `in` (mode 1).  Column x belongs to the
    // rank j with xs[j] <= x < xs[j + 1]; its value at line index k of outer
    // index o is col[j][((zs + o) * nl + k) * pitch[j] + x - xs[j]].
    struct Peers {
        void* col[8];
        int xs[9];
        int64_t pitch[8];
        int n, zs, nl;
    } peers;
};

enum { COL_TILE_DEFAULT = 0, COL_TILE_256 = 1, COL_TILE_128 = 2 };

// The last-direction pass along x (rows contiguous in memory): forward DFT of
// each row, Green's multiply (STD) or curl and Green's multiply (ROT, three
// components), inverse DFT, in place.
struct RowFusedArgs {
    const void* in;
    void* out;
    int n1, n2;                  // rows (i1, i2), i1 < n1 fastest
    int nin, nout;               // loaded / stored extent along the row (zero beyond nin)
    int64_t s1, s2, cstr;        // element strides of the rows and of a component
    const void* tws;             // later-stage twiddle table of the L-point DFT
    const void* green;           // folded Green's spectrum; x folded at L
    int64_t g1, g2;              // its strides along i1, i2 (rows of at least L/2 + 4 values)
    int f1, f2;                  // fold lengths along i1, i2 (0 = none)
    // ROT: curl symbols (as in ColArgs), the directions of i1 and i2, and the
    // Nyquist index of every direction (the index whose negation is itself)
    const void* ksym;
    int kstr;
    int ax1, ax2;
    int nyq[3];
    // L2 prefetch of a later block's rows (ROT rows; nbox = 0: none).  Map
    // dims: 8-byte units along the row, i1, i2, component
    Prefetch pf;
};

struct RowArgs {
    const void* in;
    void* out;
    int nrows;              // rows per component
    int n1;                 // rows are (i1, i2) with i1 < n1
    int nin;                // r2c: real inputs (<= L); c2r: complex inputs (L/2+1)
    int nout;               // r2c: complex outputs kept; c2r: reals kept
    int64_t in_s1, in_s2, in_cstr;   // element strides of rows (i1, i2) and component
    int64_t out_s1, out_s2, out_cstr;
    int in_f64, out_f64;
    const void* tw;         // W_L^q, q < L (L = 2 * Lh): the real-to-half-length split
    const void* tws;        // later-stage twiddle table of the Lh-point DFT (fast_stage_table)
    // r2r rows (DCT / DST I-IV through an M-point complex DFT of the extended row)
    int kind;               // LineKind of the transform
    int n;                  // FFTW size n_in
    int nstore;             // outputs written (before post-processing)
    int postpro, nfftw;     // PostPro bits and the index PP_ENFORCE_PERIOD copies from 0
    int fi, fo;             // first input / output element of the transform in its row (half-length DCT kinds)
    int ilast;              // the row element PP_NULL_LAST sets to zero (the output line's last)
    const void* tw2;        // W_{2M}^q, q < 2M (pre/post twiddles of the r2r kinds)
    Prefetch pf;            // r2c / c2r rows
};

// Fills `pf` for a 4-D view of 8-byte units (dims[0] fastest; strides in
// bytes of dims 1..3) with box `box`; false (pf.nbox = 0) when the view does
// not meet the tensor-map rules (16-byte aligned base and strides).
bool make_prefetch(Prefetch& pf, const void* base, const uint64_t dims[4], const uint64_t strides[3], const uint32_t box[4],
                   int nbox, int step, int dist);

bool fast_col_supported(int L);
// columns per CTA of a column c2c pass of length L with CTA tile `tile`
int fast_col_tile_width(int f64, int L, int tile);
// rows per CTA of the r2c / c2r row pass of real length L
int fast_row_tile_rows(int f64, int L);
// row positions per block of the fused ROT rows
int fast_rowrot_rows(int f64, int L);
bool fast_row_supported(int L);

// First radix of the register DFTs for an n-point line: 32 in FP32 and 16 in
// FP64 for powers of two; 24 (3 x 8) in FP32 and 12 (3 x 4) in FP64 for 3 x 2^k.
__host__ __device__ constexpr int fast_radix1_of(int n, int f64) {
    return (n % 3 == 0) ? (f64 ? 12 : 24) : (f64 ? 16 : 32);
}
int fast_radix1(int f64, int n);
// First radices that differ from fast_radix1_of (the tables of those passes
// are built with the same functions):
//  - FP32 384- and 768-point lines of the forward / inverse columns and the
//    rows: 48 (3 x 16), two Stockham stages instead of three (768-point
//    columns 0.62 -> 0.56 ms along y, 0.87 -> 0.72 ms along z at 384^3);
//  - FP64 power-of-two lines of the column passes (modes 0, 1, 2) and of the
//    rows: 32, one exchange per transform instead of two, up to 255 registers
//    in two 128-thread CTAs per SM (512^3: fused 5.97 -> 4.47 ms, y passes
//    1.57 / 1.65 -> 1.24 / 1.37 ms in a standalone driver); 3 x 2^k lines keep
//    12 (a first radix of 24 spills 184 bytes in the fused pass).
__host__ __device__ constexpr bool fast_radix48(int n, int f64) { return !f64 && (n == 384 || n == 768); }
// rows: n is the half-length DFT of the r2c / c2r split
__host__ __device__ constexpr int fast_radix1_row(int n, int f64) {
    return fast_radix48(n, f64) ? 48 : ((f64 && n % 3 != 0) ? 32 : fast_radix1_of(n, f64));
}
// column c2c passes of mode 0 (forward), 1 (inverse), 2 (fused) or 3 (fused
// ROT); radix 48 not used by the fused passes
__host__ __device__ constexpr int fast_radix1_mode(int n, int f64, int mode) {
    return (mode < 2 && fast_radix48(n, f64)) ? 48 : ((n % 3 != 0) ? fast_radix1_of(n, 0) : fast_radix1_of(n, f64));
}
// the real-side columns (col_real_kernel, col_real_pair_kernel): FP32
// power-of-two lines from 128 to FLB_COLREAL_R16_MAX points take a first radix
// of 16 (half the registers of 32, four 256-thread CTAs per SM), else the
// default (256-point y columns of the 513 x 257 x 257 node grid: r2c 73.6 ->
// 64.6 us, c2r 68.1 -> 66.7 us; the 64 x 128^3 batch 3.19 -> 3.05 ms)
#ifndef FLB_COLREAL_R16_MAX
#define FLB_COLREAL_R16_MAX 256
#endif
__host__ __device__ constexpr int fast_radix1_colreal(int n, int f64) {
    return (!f64 && n % 3 != 0 && n >= 128 && n <= FLB_COLREAL_R16_MAX) ? 16 : fast_radix1_of(n, f64);
}
// the fused ROT rows (row_rot_kernel): FP32 384- and 768-point lines with a first
// radix of 48 (two Stockham stages, one exchange per DFT instead of two; 168
// registers, 28 bytes spilled), else the fused passes' radix
#ifndef FLB_ROWROT_R48
#define FLB_ROWROT_R48 1
#endif
// the fused rows (row_fused_kernel, row_rot_kernel) of FP64 3 x 2^k lines:
// a first radix of 24 (P = n / 24 lanes per row, so lines up to 768 points
// fit one warp and the x-last order applies), else the fused passes' radix
#ifndef FLB_ROWF64_R24
#define FLB_ROWF64_R24 1
#endif
__host__ __device__ constexpr int fast_radix1_rowfused(int n, int f64) {
    return (FLB_ROWF64_R24 && f64 && n % 3 == 0 && n % 24 == 0 && n / 24 <= 32 && n / 24 >= 2) ? 24 : fast_radix1_mode(n, f64, 2);
}
__host__ __device__ constexpr int fast_radix1_rowrot(int n, int f64) {
    return (FLB_ROWROT_R48 && fast_radix48(n, f64)) ? 48 : fast_radix1_rowfused(n, f64);
}
// the half-length DCT / DST rows (row_dct_kernel): the LH-point DFT's first
// radix.  FP32 power-of-two lines up to 256 points take 16 (16 complex values
// per lane, 64 registers, four 256-thread CTAs per SM: 513 x 257 x 257 node
// grid, DCT-III rows 0.167 -> 0.134 ms, DCT-II rows 0.134 -> 0.115 ms against
// a first radix of 32 at two CTAs per SM); FLB_DCT_R1 / FLB_DCT_R1_F64 set
// the FP32 / FP64 radix of the power-of-two lines it divides (0: the column
// passes' radix).
#ifndef FLB_DCT_R1
#define FLB_DCT_R1 16
#endif
#ifndef FLB_DCT_R1_F64
#define FLB_DCT_R1_F64 0
#endif
__host__ __device__ constexpr int fast_radix1_dct(int lh, int f64) {
    return ((f64 ? FLB_DCT_R1_F64 : FLB_DCT_R1) > 0 && lh % 3 != 0 && lh % (f64 ? FLB_DCT_R1_F64 : FLB_DCT_R1) == 0 &&
            lh / (f64 ? FLB_DCT_R1_F64 : FLB_DCT_R1) <= 16)
               ? (f64 ? FLB_DCT_R1_F64 : FLB_DCT_R1)
               : fast_radix1_of(lh, f64);
}
// radix of a later Stockham stage: the largest common divisor of what is left
// of the line (n / Ns) and the first radix
__host__ __device__ constexpr int fast_gcd(int a, int b) { return b == 0 ? a : fast_gcd(b, a % b); }
// Complex entries of the later-stage twiddle table of an n-point register DFT
// (first radix of the default passes, or r1).
int fast_stage_table_len(int n, int f64);
int fast_stage_table_len_r1(int n, int r1);
// Entry e of that table is W_M^q = exp(-2 pi i q / M); sets q and M.
// Layout: one block of n entries per stage after the first (Ns = r1, r1*Rs, ...
// with Rs = gcd(n/Ns, r1)); in a block, pair (b * Rs/2 + rp) * P + p (P = n/r1)
// holds W_{Ns Rs}^{r k} for r = 2rp, 2rp+1 and k = (p + P b) mod Ns: the
// twiddles of butterfly b of thread p, two per 16-byte (FP32) load.
__host__ __device__ inline void fast_stage_exponent(int n, int r1, int e, int* q, int* M) {
    const int P = n / r1;
    const int s = e / n, w = e % n;
    int Ns = r1;
    for (int i = 0; i < s; ++i) Ns *= fast_gcd(n / Ns, r1);
    const int Rs = fast_gcd(n / Ns, r1);
    const int pair = w / 2, half = w % 2;
    const int p = pair % P, t = pair / P;
    const int rp = t % (Rs / 2), b = t / (Rs / 2);
    const int r = 2 * rp + half, k = (p + P * b) % Ns;
    *M = Ns * Rs;
    *q = (int)(((long long)r * k) % (Ns * Rs));
}

// column c2c pass of mode 0 (forward DFT), 1 (inverse DFT), 2 (forward,
// Green's multiply, inverse) or 3 (forward, curl and Green's multiply of
// groups of three components, inverse)
cudaError_t launch_fast_col(int f64, int mode, int L, const ColArgs& a, int ncomp, cudaStream_t s);
// fused pass along x rows: lengths whose line fits in one warp
bool fast_rowfused_supported(int f64, int L);
// rot: three components per row position (curl and Green's multiply), else STD
cudaError_t launch_fast_rowfused(int f64, int rot, int L, const RowFusedArgs& a, int ncomp, cudaStream_t s);
cudaError_t launch_fast_row(int f64, int c2r, int L, const RowArgs& a, int ncomp, cudaStream_t s);
// r2r rows (DCT / DST I-IV) through an M-point complex register DFT
bool fast_r2r_supported(int M);
// DCT / DST II-IV rows of even length n (M = 2n) that run through one
// n/2-point register DFT instead: the family (2, 3 or 4); DCT-I / DST-I rows
// (M = 2(n - 1) / 2(n + 1)) through one M/2-point register DFT: family 1;
// else 0.  Their tables, with N = fast_dct_length (n, or M for family 1):
// tw = W_N^q (q < N), tws = the stage table of the N/2-point DFT, tw2 =
// W_2M^q as for the M-point kernel.
int fast_dct_family(int kind, int n, int M);
int fast_dct_length(int kind, int n, int M);
// launches the half-length kernel when fast_dct_family(a.kind, a.n, M) != 0
cudaError_t launch_fast_r2r(int f64, int M, const RowArgs& a, int ncomp, cudaStream_t s);
// column r2c (c2r = 0: real in, X[0..L/2] out) and c2r (c2r = 1)
cudaError_t launch_fast_colreal(int f64, int c2r, int L, const ColArgs& a, int ncomp, cudaStream_t s);

}  // namespace flb
