// Entry points of oracle/_ref/libflups_ref.so: the reference's own solver
// (its src/*.cpp, compiled unmodified against this directory's FFTW, MPI
// and h3lpr stand-ins) called through its public C API (src/flups.h:
// flups_topo_new, flups_init, flups_set_greenType, flups_set_alpha,
// flups_setup, flups_solve, flups_cleanup), on one rank.  Dense arrays in
// (lda, n2, n1, n0) order with the x index fastest are copied into and out
// of the reference's user topology (axis 0, flups_locID layout).  Test
// infrastructure of the oracle: a checker and the CPU baseline, never the
// product.  Only the symbols below are exported (the library is built with
// hidden visibility and -Bsymbolic, so the reference's flups_* names stay
// private to it).
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "flups.h"

#define FLB_REF_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

struct Case {
    FLUPS_Topology* topo = nullptr;
    FLUPS_Solver* solver = nullptr;
    double* field = nullptr;
    double* rhs = nullptr;
    int lda = 1, n[3] = {0, 0, 0}, nmem[3] = {0, 0, 0};
};

void pack(const Case& c, const double* dense, double* topo_arr) {
    for (int l = 0; l < c.lda; ++l)
        for (int i2 = 0; i2 < c.n[2]; ++i2)
            for (int i1 = 0; i1 < c.n[1]; ++i1)
                for (int i0 = 0; i0 < c.n[0]; ++i0)
                    topo_arr[flups_locID(0, i0, i1, i2, l, 0, c.nmem, 1)] =
                        dense[(((size_t)l * c.n[2] + i2) * c.n[1] + i1) * c.n[0] + i0];
}

void unpack(const Case& c, const double* topo_arr, double* dense) {
    for (int l = 0; l < c.lda; ++l)
        for (int i2 = 0; i2 < c.n[2]; ++i2)
            for (int i1 = 0; i1 < c.n[1]; ++i1)
                for (int i0 = 0; i0 < c.n[0]; ++i0)
                    dense[(((size_t)l * c.n[2] + i2) * c.n[1] + i1) * c.n[0] + i0] =
                        topo_arr[flups_locID(0, i0, i1, i2, l, 0, c.nmem, 1)];
}

}  // namespace

// Sets up a reference solver.  bcs: [dir][side][lda] boundary types;
// center: [3] centring; green: the kernel (FLUPS_GreenType); alpha <= 0
// keeps the reference's default; odiff: FLUPS_DiffType.  Returns a handle.
FLB_REF_EXPORT void* flups_ref_new(const int nglob[3], int lda, const int* bcs, const double h[3], const double L[3],
                                   const int center[3], int green, double alpha, int odiff) {
    Case* c = new Case;
    c->lda = lda;
    const int nproc[3] = {1, 1, 1}, axproc[3] = {0, 1, 2};
    c->topo = flups_topo_new(0, lda, nglob, nproc, false, axproc, FLUPS_ALIGNMENT, MPI_COMM_WORLD);
    std::vector<FLUPS_BoundaryType> store(6 * (size_t)lda);
    FLUPS_BoundaryType* bc[3][2];
    for (int d = 0; d < 3; ++d)
        for (int s = 0; s < 2; ++s) {
            bc[d][s] = store.data() + (2 * d + s) * lda;
            for (int l = 0; l < lda; ++l) bc[d][s][l] = (FLUPS_BoundaryType)bcs[(2 * d + s) * lda + l];
        }
    const FLUPS_CenterType ct[3] = {(FLUPS_CenterType)center[0], (FLUPS_CenterType)center[1], (FLUPS_CenterType)center[2]};
    c->solver = flups_init(c->topo, bc, h, L, (FLUPS_DiffType)odiff, ct);
    flups_set_greenType(c->solver, (FLUPS_GreenType)green);
    if (alpha > 0) flups_set_alpha(c->solver, alpha);
    flups_setup(c->solver, true);
    for (int d = 0; d < 3; ++d) {
        c->n[d] = flups_topo_get_nloc(c->topo, d);
        c->nmem[d] = flups_topo_get_nmem(c->topo, d);
    }
    const size_t mem = flups_topo_get_memsize(c->topo);
    c->field = (double*)flups_malloc(sizeof(double) * mem);
    c->rhs = (double*)flups_malloc(sizeof(double) * mem);
    memset(c->field, 0, sizeof(double) * mem);
    memset(c->rhs, 0, sizeof(double) * mem);
    return c;
}

// One solve: rhs_dense -> field_dense (both lda x n2 x n1 x n0, x fastest).
// type: FLUPS_SolverType (STD / ROT).  Returns the wall time of the
// flups_solve call in seconds (the copies into and out of the reference's
// layout are outside it).
FLB_REF_EXPORT double flups_ref_solve(void* h, const double* rhs_dense, double* field_dense, int type) {
    Case* c = static_cast<Case*>(h);
    pack(*c, rhs_dense, c->rhs);
    const auto t0 = std::chrono::steady_clock::now();
    flups_solve(c->solver, c->field, c->rhs, (FLUPS_SolverType)type);
    const auto t1 = std::chrono::steady_clock::now();
    unpack(*c, c->field, field_dense);
    return std::chrono::duration<double>(t1 - t0).count();
}

FLB_REF_EXPORT void flups_ref_free(void* h) {
    Case* c = static_cast<Case*>(h);
    flups_free(c->field);
    flups_free(c->rhs);
    flups_cleanup(c->solver);
    flups_topo_free(c->topo);
    delete c;
}
