// Descriptors shared by the host planner and the CUDA line-transform kernels.
//
// One "pass" transforms every line of a 3-D (x fastest) array along one
// direction: it gathers the line (with the zero padding and the fieldstart
// shift that the reference's SwitchTopo applies, src/SwitchTopoX_a2a.cpp:
// 174-247 and src/chunk_tools.cpp:385-466), runs the 1-D transform the
// reference would hand to FFTW (src/FFTW_plan_dim.cpp:635-720), applies the
// plan's post-processing (src/FFTW_plan_dim.cpp:497-622) and scatters the
// result into the next array.  A "fused" pass runs the last forward
// transform, the spectral multiply (src/dothemagic_std.ipp:56-83,
// src/dothemagic_rot.ipp:102-350) and the first backward transform on the
// same line without a round trip through HBM.
#pragma once
#include <stdint.h>

namespace flb {

// 1-D transform kinds.  The r2r kinds are FFTW's (REDFT00 = DCT-I, ...).
enum LineKind : int {
    LK_NONE = 0,
    LK_R2C = 1,    // real -> complex, forward DFT (n_in reals -> n_in/2+1 complex)
    LK_C2R = 2,    // complex -> real, backward DFT
    LK_C2C = 3,    // complex DFT with sign
    LK_DCT1 = 10,  // REDFT00
    LK_DCT2 = 11,  // REDFT10
    LK_DCT3 = 12,  // REDFT01
    LK_DCT4 = 13,  // REDFT11
    LK_DST1 = 14,  // RODFT00
    LK_DST2 = 15,  // RODFT10
    LK_DST3 = 16,  // RODFT01
    LK_DST4 = 17,  // RODFT11
};

enum PostPro : int { PP_NONE = 0, PP_NULL_FIRST = 1, PP_NULL_LAST = 2, PP_ENFORCE_PERIOD = 4 };

constexpr int kMaxComp = 3;       // per-component transform specs (lda <= 3)
constexpr int kMaxRadices = 24;   // FFT stages

// What happens on one line of one component.
struct LineSpec {
    int kind;      // LineKind
    int sign;      // -1 forward, +1 backward (C2C only)
    int n_in;      // FFTW transform size (reals for r2r/r2c/c2r, complex for c2c)
    int fi, fo;    // fftwstart_in / fftwstart_out
    int postpro;   // PostPro bit set
    int nfftw;     // index copied from 0 for PP_ENFORCE_PERIOD
};

// One direction's transform of every line.
struct LineStage {
    LineSpec spec[kMaxComp];
    int M;                       // complex FFT length
    int nrad;                    // number of Stockham stages
    int radix[kMaxRadices];
    int n_b;                     // length of the padded input line (input-transform units)
    int fieldstart;              // placement of the source line in the padded line
    int n_o;                     // length of the output line (output-transform units)
    int in_cplx, out_cplx;       // element type before / after the transform
    int store_off, n_store;      // part of the output line kept
    const void* tw;              // W_{2M}^q, q in [0, 2M), working precision (complex)
};

// Spectral multiply fused between two stages.
struct MultSpec {
    int mode;                   // 0 none, 1 STD (G * normfact), 2 ROT (curl then G * normfact)
    const void* green;          // folded real Green's spectrum, working precision
    int64_t gstr[3];            // element strides of the folded Green array (x fastest)
    int gfold[3];               // DFT length for folding (i -> min(i, M - i)), 0 = no folding
    int gn[3];                  // folded extents (bounds)
    double normfact;
    // ROT: wave numbers k = (is + koffset) * kfact_c, complex kfact per (dir, comp)
    double koffset[3];
    double symstart[3];
    double kfact[3][3][2];
    double hgrid[3];
    int odiff;                  // 1 SPE, 2 FD2, 4 FD4, 6 FD6
};

// Launch arguments of one pass.
struct PassArgs {
    int axis;                    // direction transformed (0 = x)
    int n_src;                   // extent of the source line (source elements)
    int n_a, n_b;                // extents of the two other directions (a is the faster one)
    int ncomp;                   // components (x batch) per line position
    int lda;                     // spec index = comp % lda
    int64_t in_str[3], in_cstr;  // element strides of the source array
    int64_t out_str[3], out_cstr;
    const void* in;
    void* out;
    int lines_per_cta;
    int fused;                   // 0: one stage; 1: stage0 -> multiply -> stage1
    int comps_together;          // ROT: the three components of a position in one CTA
    LineStage st[2];
    MultSpec mult;
    int nlines;                  // number of line positions (n_a * n_b)
};

}  // namespace flb
