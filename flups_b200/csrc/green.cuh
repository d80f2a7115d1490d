// FP64 Green's-function setup on the device.
//
// The kernels and their splittings follow the reference's
// src/green_kernels.hpp:26-773 and src/green_functions.cpp:27-708; the
// special functions follow the published methods the reference cites
// (Numerical Recipes 3rd ed. 6.5.1 for K0/K1, Chebyshev fits of E1, the
// GalSim Chebyshev-Pade fits of Si, Humbert's series for Ji0c, the
// closed-form 1-D lattice Green's function of the 3-point stencil).
#pragma once
#include <stdint.h>

namespace flb {

enum GreenKind : int {
    G_CHAT_2 = 0, G_LGF_2 = 1, G_HEJ_2 = 2, G_HEJ_4 = 3, G_HEJ_6 = 4, G_HEJ_8 = 5, G_HEJ_10 = 6, G_HEJ_0 = 7,
    G_LGF_4 = 8, G_LGF_6 = 9, G_LGF_8 = 10, G_MEHR_4L = 11, G_MEHR_6L = 12, G_MEHR_4F = 13, G_MEHR_6F = 14,
};

// Far-field expansion: sum_t coef_t n1^a n2^b n3^c n^e  + logc * log(n)
struct FarTerm {
    double coef;   // coefficient times pi^p
    int a, b, c, e;
};

struct GreenEvalArgs {
    int kind;
    int nunb;                 // 3, 2, 1 or 0 unbounded directions
    int size[3];              // extents of the Green's topology 0 (x fastest)
    int cplx;                 // complex storage (only real parts written)
    int ax[3];                // topology axis order (ax0 = first Green plan's direction)
    double symstart[3], hfact[3], kfact[3], koffset[3];
    double length;            // HEJ smoothing length (alpha h) or h/pi for HEJ_0
    double hgrid;             // grid spacing (LGF)
    double r_eq2d, r_cut, k_cut;
    double g0;                // value at r = 0 (3 unbounded, non-LGF)
    int set_g0;
    int chat2d_origin;        // 2 unbounded CHAT_2: special value at the origin
    const double* table;      // LGF/MEHR table (32^3 or 32^2)
    int tableN;
    const FarTerm* far;
    int nfar;
    double far_log;
    double* out;
    // canonical box: with 3 unbounded directions the function depends on |is|
    // only, so only indices up to symstart are evaluated and a second kernel
    // copies them to their mirror images
    int canon;
    int csize[3];
};

struct GreenFinalArgs {
    // final spectral Green (double, complex or real) -> folded working-precision array
    const double* spec;
    int spec_cplx;
    int spec_n[3];            // spectral extents (x fastest)
    int fold_n[3];            // folded extents
    int64_t fold_str[3];
    double volfact;
    int complete;             // 2-unbounded + 1-spectral completion with the 3-spectral kernel
    int spec_dim;             // spectral direction of that completion
    int kind;
    double kfact[3], koffset[3], symstart[3];
    int ax[3];
    double hgrid, length;
    int reset0;               // set the (0,0,0) mode to zero
    double scale;             // the solver's normalisation, folded into the stored spectrum
    void* out;
    int out_f64;
};

}  // namespace flb
