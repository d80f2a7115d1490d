// Per-direction transform tables: which 1-D transform each direction needs,
// its sizes, offsets, wave-number factors and post-processing.  Restates
// FFTW_plan_dim (src/FFTW_plan_dim.cpp:35-209) and its cell/node initialisers
// (src/FFTW_plan_dim_cell.cpp:19-390, src/FFTW_plan_dim_node.cpp:19-461).
#include <algorithm>
#include <cmath>

#include "host.hpp"

namespace flb {

static const double kTwoPi = 2.0 * M_PI;

DirPlan::DirPlan(int lda_, int dim_, const double h[3], const double L[3], const int bcl[3], const int bcr[3], int sign_, bool green,
                 int center_)
    : lda(lda_), dim(dim_), sign(sign_), is_green(green), center(center_) {
    FLB_CHECK(dim >= 0 && dim < 3, "we are only creating plans on dim from 0 to 2");
    for (int c = 0; c < lda; ++c) {
        bc[0][c] = bcl[c];
        bc[1][c] = bcr[c];
    }
    // FFTW_plan_dim.cpp:108-139: the type is the sum of the BCs of component 0
    const int t = bc[0][0] + bc[1][0];
    if (t <= SYMSYM) {
        type = SYMSYM; volfact = 1.0; kfact = kTwoPi / (2.0 * L[dim]); is_spectral = green;
    } else if (t <= MIXUNB) {
        type = MIXUNB; volfact = h[dim]; kfact = kTwoPi / (4.0 * L[dim]);
    } else if (t == PERPER) {
        type = PERPER; volfact = 1.0; kfact = kTwoPi / L[dim]; is_spectral = green;
    } else if (t == UNBUNB) {
        type = UNBUNB; volfact = h[dim]; kfact = kTwoPi / (2.0 * L[dim]);
    } else if (t == EMPTY) {
        type = EMPTY; volfact = 1.0; kfact = 0.0;
    } else {
        FLB_CHECK(false, "Invalid combination of BCs");
    }
    for (int c = 0; c < lda; ++c)
        FLB_CHECK(bc[0][c] + bc[1][c] <= type, "dimension %d's bc = %d %d is not compatible with the plan choosen = %d", c,
                  bc[0][c], bc[1][c], type);
}

void DirPlan::init(const int size[3], bool is_complex) {
    const int n = size[dim];
    const bool cell = (center == CELL_CENTER);
    if (type == SYMSYM) {
        FLB_CHECK(!is_complex, "the data cannot be complex");
        bool t4 = bc[0][0] != bc[1][0];
        for (int c = 1; c < lda; ++c)
            FLB_CHECK((bc[0][c] != bc[1][c]) == t4,
                      "one component has an EVEN-ODD condition, while one of the other uses EVEN-EVEN or ODD-ODD, which is not supported");
        cell ? r2r_cell(n) : r2r_node(n);
    } else if (type == MIXUNB) {
        FLB_CHECK(!is_complex, "the data cannot be complex");
        cell ? mix_cell(n) : mix_node(n);
    } else if (type == PERPER) {
        cell ? per_cell(n, is_complex) : per_node(n, is_complex);
    } else if (type == UNBUNB) {
        cell ? unb_cell(n, is_complex) : unb_node(n, is_complex);
    }
}

// ------------------------------------------------------------------ cell
void DirPlan::r2r_cell(int n) {
    symstart = 0; fieldstart = 0; isr2c = false;
    normfact *= 1.0 / (2.0 * n);
    for (int c = 0; c < lda; ++c) {
        const int l = bc[0][c], r = bc[1][c];
        if (is_green) {
            postpro[c] = 0; fstart_in[c] = fstart_out[c] = 0; imult[c] = false;
            if (l != r) { n_in[c] = n; n_out = n; koffset = 0.5; }
            else { n_in[c] = n; n_out = n + 1; koffset = 0.0; }
            return;
        }
        n_in[c] = n;
        if (l == EVEN) {
            imult[c] = false;
            if (r == EVEN) {
                n_out = n + 1; koffset = 0.0;
                fstart_in[c] = fstart_out[c] = 0;
                if (sign == FLUPS_FORWARD) { kind[c] = REDFT10; postpro[c] = PP_NULL_LAST; }
                else { kind[c] = REDFT01; postpro[c] = PP_NONE; }
            } else if (r == ODD) {
                n_out = n; koffset = 0.5;
                kind[c] = REDFT11; fstart_in[c] = fstart_out[c] = 0; postpro[c] = PP_NONE;
            } else {
                FLB_CHECK(false, "unable to init the solver required");
            }
        } else if (l == ODD) {
            imult[c] = true;
            if (r == ODD) {
                n_out = n + 1; koffset = 0.0;
                if (sign == FLUPS_FORWARD) { kind[c] = RODFT10; fstart_in[c] = 0; fstart_out[c] = 1; postpro[c] = PP_NULL_FIRST; }
                else { kind[c] = RODFT01; fstart_in[c] = 1; fstart_out[c] = 0; postpro[c] = PP_NULL_LAST; }
            } else if (r == EVEN) {
                n_out = n; koffset = 0.5;
                kind[c] = RODFT11; fstart_in[c] = fstart_out[c] = 0; postpro[c] = PP_NONE;
            } else {
                FLB_CHECK(false, "unable to init the solver required");
            }
        } else {
            FLB_CHECK(false, "unable to init the solver required");
        }
    }
}

void DirPlan::mix_cell(int n) {
    isr2c = false;
    if (is_green) fieldstart = 0;
    else if (bc[0][0] == UNB) fieldstart = n;
    else if (bc[1][0] == UNB) fieldstart = 0;
    symstart = 0;
    normfact *= 1.0 / (4.0 * n);
    for (int c = 0; c < lda; ++c) {
        const int l = bc[0][c], r = bc[1][c];
        if (is_green) {
            n_in[c] = 2 * n + 1; n_out = 2 * n + 1; koffset = 0.0;
            fstart_in[c] = fstart_out[c] = 0; postpro[c] = PP_NONE; imult[c] = false; kind[c] = REDFT00;
            continue;
        }
        n_in[c] = 2 * n; n_out = 2 * n + 1; koffset = 0.0;
        if ((l == EVEN && r == UNB) || (l == UNB && r == EVEN)) {
            imult[c] = false; fstart_in[c] = fstart_out[c] = 0;
            if (sign == FLUPS_FORWARD) { kind[c] = REDFT10; postpro[c] = PP_NULL_LAST; }
            else { kind[c] = REDFT01; postpro[c] = PP_NONE; }
        } else if ((l == UNB && r == ODD) || (l == ODD && r == UNB)) {
            imult[c] = true;
            if (sign == FLUPS_FORWARD) { kind[c] = RODFT10; fstart_in[c] = 0; fstart_out[c] = 1; postpro[c] = PP_NULL_FIRST; }
            else { kind[c] = RODFT01; fstart_in[c] = 1; fstart_out[c] = 0; postpro[c] = PP_NULL_LAST; }
        } else {
            FLB_CHECK(false, "unable to init the solver required");
        }
    }
}

void DirPlan::per_cell(int n, bool c) {
    // only n_in[0] is set: DFT plans use it alone (FFTW_plan_dim_cell.cpp:301-343)
    if (c) { n_in[0] = n; n_out = n; isr2c = false; }
    else { n_in[0] = n; n_out = n / 2 + 1; isr2c = true; }
    fieldstart = 0;
    symstart = c ? n / 2.0 : 0.0;
    normfact *= 1.0 / n;
    for (int k = 0; k < lda; ++k) { postpro[k] = PP_NONE; fstart_in[k] = fstart_out[k] = 0; imult[k] = false; }
}

void DirPlan::unb_cell(int n, bool c) {
    if (c) { n_in[0] = 2 * n; n_out = 2 * n; isr2c = false; }
    else { n_in[0] = 2 * n; n_out = n + 1; isr2c = true; }
    fieldstart = 0;
    symstart = n;
    normfact *= 1.0 / (2.0 * n);
    for (int k = 0; k < lda; ++k) { fstart_in[k] = fstart_out[k] = 0; postpro[k] = PP_NONE; imult[k] = false; }
}

// ------------------------------------------------------------------ node
void DirPlan::r2r_node(int n) {
    symstart = 0; fieldstart = 0; isr2c = false;
    normfact *= 1.0 / (2.0 * (n - 1));
    for (int c = 0; c < lda; ++c) {
        const int l = bc[0][c], r = bc[1][c];
        if (is_green) {
            postpro[c] = 0; fstart_in[c] = fstart_out[c] = 0; imult[c] = false;
            if (l == EVEN && r == EVEN) { n_in[c] = n; n_out = n; koffset = 0.0; }
            else if (l == EVEN && r == ODD) { n_in[c] = n - 1; n_out = n; koffset = 0.5; }
            else if (l == ODD && r == ODD) { n_in[c] = n - 2; n_out = n; koffset = 0.0; }
            else if (l == ODD && r == EVEN) { n_in[c] = n - 1; n_out = n; koffset = 0.5; }
            return;
        }
        if (l == EVEN) {
            imult[c] = false;
            if (r == EVEN) {
                n_in[c] = n; n_out = n; postpro[c] = PP_NONE; koffset = 0.0; kind[c] = REDFT00;
                fstart_in[c] = fstart_out[c] = 0;
            } else if (r == ODD) {
                n_in[c] = n - 1; n_out = n; koffset = 0.5; fstart_in[c] = fstart_out[c] = 0;
                kind[c] = (sign == FLUPS_FORWARD) ? REDFT01 : REDFT10;
                postpro[c] = PP_NULL_LAST;
            } else {
                FLB_CHECK(false, "unable to init the solver required");
            }
        } else if (l == ODD) {
            imult[c] = true;
            if (r == ODD) {
                n_in[c] = n - 2; n_out = n; koffset = 0.0; fieldstart = 0;
                kind[c] = RODFT00; fstart_in[c] = fstart_out[c] = 1; postpro[c] = PP_NULL_FIRST + PP_NULL_LAST;
            } else if (r == EVEN) {
                n_in[c] = n - 1; n_out = n; koffset = 0.5; fieldstart = 0;
                if (sign == FLUPS_FORWARD) { kind[c] = RODFT01; fstart_in[c] = 1; fstart_out[c] = 0; postpro[c] = PP_NULL_LAST; }
                else { kind[c] = RODFT10; fstart_in[c] = 0; fstart_out[c] = 1; postpro[c] = PP_NULL_FIRST; }
            } else {
                FLB_CHECK(false, "unable to init the solver required");
            }
        } else {
            FLB_CHECK(false, "unable to init the solver required");
        }
    }
}

void DirPlan::mix_node(int n) {
    isr2c = false;
    if (is_green) fieldstart = 0;
    else if (bc[0][0] == UNB) fieldstart = n - 1;
    else if (bc[1][0] == UNB) fieldstart = 0;
    symstart = 0;
    normfact *= 1.0 / (2.0 * ((2 * n - 1) - 1.0));
    for (int c = 0; c < lda; ++c) {
        const int l = bc[0][c], r = bc[1][c];
        const bool eu = (l == EVEN && r == UNB) || (l == UNB && r == EVEN);
        const bool ou = (l == UNB && r == ODD) || (l == ODD && r == UNB);
        if (is_green) {
            if (eu || ou) { n_in[c] = 2 * n - 1; n_out = n_in[c]; koffset = 0.0; }
            fstart_in[c] = fstart_out[c] = 0; postpro[c] = PP_NONE; imult[c] = false; kind[c] = REDFT00;
            continue;
        }
        if (eu) {
            n_in[c] = 2 * n - 1; n_out = n_in[c]; koffset = 0.0;
            fstart_in[c] = fstart_out[c] = 0; postpro[c] = PP_NONE; imult[c] = false; kind[c] = REDFT00;
        } else if (ou) {
            n_in[c] = (2 * n - 1) - 2; n_out = n_in[c] + 2; koffset = 0.0; imult[c] = true;
            kind[c] = RODFT00; fstart_in[c] = fstart_out[c] = 1; postpro[c] = PP_NULL_FIRST + PP_NULL_LAST;
        } else {
            FLB_CHECK(false, "unable to init the solver required");
        }
    }
}

void DirPlan::per_node(int n, bool c) {
    for (int k = 0; k < lda; ++k) n_in[k] = n - 1;
    if (c) { n_out = n; isr2c = false; }
    else { n_out = n_in[0] / 2 + 1 + 1; isr2c = true; }
    fieldstart = 0;
    symstart = c ? (n - 1) / 2.0 : 0.0;
    normfact *= 1.0 / (n - 1);
    for (int k = 0; k < lda; ++k) { postpro[k] = PP_ENFORCE_PERIOD; fstart_in[k] = fstart_out[k] = 0; imult[k] = false; }
}

void DirPlan::unb_node(int n, bool c) {
    if (c) { n_in[0] = 2 * (n - 1); n_out = 2 * (n - 1); isr2c = false; }
    else { n_in[0] = 2 * (n - 1); n_out = n_in[0] / 2 + 1; isr2c = true; }
    fieldstart = 0;
    symstart = n - 1;
    normfact *= 1.0 / (2.0 * (n - 1));
    for (int k = 0; k < lda; ++k) { postpro[k] = PP_NONE; fstart_in[k] = fstart_out[k] = 0; imult[k] = false; }
}

// stable sort of the three directions by plan type (src/FFTW_plan_dim.cpp:35-51)
void sort_plans(DirPlan p[3]) {
    DirPlan tmp[3] = {p[0], p[1], p[2]};
    int order[3] = {0, 1, 2};
    std::stable_sort(order, order + 3, [&](int a, int b) { return tmp[a].type < tmp[b].type; });
    for (int i = 0; i < 3; ++i) p[i] = tmp[order[i]];
}

}  // namespace flb
