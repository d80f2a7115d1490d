/*
 * flups.h -- C ABI of the B200-native FLUPS solve path (libflups_b200.so).
 *
 * Every entry point keeps the name, signature and meaning of the reference's
 * C API (vortexlab-uclouvain/flups, src/flups.h); the comment above each one
 * cites the declaration it replaces.  The solver runs on one CUDA device with
 * a size-1 communicator.  Differences a caller can see:
 *   - rhs/field of flups_solve may be host or device pointers (detected per
 *     call); flups_get_innerBuffer returns CUDA managed memory (host code
 *     and kernels may both use it) and the spectral inner topology is x
 *     fastest (axis 0), complex, rows padded to 8 complex;
 *   - flups_set_stream takes a cudaStream_t (the reference ignores it);
 *   - programmer errors abort with a message, as FLUPS_CHECK does;
 *   - additive entry points (precision, batching, errors) live in
 *     flups_b200.h.
 */
#ifndef FLUPS_H
#define FLUPS_H

#include <stddef.h>
#include <stdint.h>

#include "flups_interface.h"
#include "flups_mpi.h"

#ifdef __cplusplus
#include <cmath>
extern "C" {
#else
#include <math.h>
#include <stdbool.h>
#endif

typedef struct Solver FLUPS_Solver;
typedef struct Topology FLUPS_Topology;
typedef struct Profiler FLUPS_Profiler;

typedef enum BoundaryType FLUPS_BoundaryType;
typedef enum GreenType FLUPS_GreenType;
typedef enum SolverType FLUPS_SolverType;
typedef enum DiffType FLUPS_DiffType;
typedef enum CenterType FLUPS_CenterType;

/* ---------------------------------------------------------------- memory */
/* src/flups.h:51 -- aligned host allocation (zeroed) */
void* flups_malloc(size_t size);
/* src/flups.h:61 */
void flups_free(void* data);
/* src/flups.h:69 -- writes <exe>.flups.info with the build settings */
void flups_info(int argc, char** argv);

/* src/flups.h:109-119 -- memory index of (i0,i1,i2) given in axsrc order, for an array in axtrg order */
static inline size_t flups_locID(const int axsrc, const int i0, const int i1, const int i2, const int lia, const int axtrg,
                                 const int size[3], const int nf) {
    const int idx[3] = {i0, i1, i2};
    const int d0 = (3 + axtrg - axsrc) % 3;
    const int a0 = axtrg, a1 = (axtrg + 1) % 3, a2 = (axtrg + 2) % 3;
    return (size_t)idx[d0] * nf +
           (size_t)size[a0] * nf * ((size_t)idx[(d0 + 1) % 3] + (size_t)size[a1] * ((size_t)idx[(d0 + 2) % 3] + (size_t)lia * size[a2]));
}

/* src/flups.h:170-184 -- symmetrised spectral index (absolute value) in axtrg order */
static inline void flups_symID(const int axsrc, const int i0, const int i1, const int i2, const int istart[3],
                               const double symstart[3], const int axtrg, int is[3]) {
    const int ie[3] = {istart[axsrc] + i0, istart[(axsrc + 1) % 3] + i1, istart[(axsrc + 2) % 3] + i2};
    const int d0 = (3 + axtrg - axsrc) % 3;
    for (int k = 0; k < 3; ++k) {
        const int ax = (axtrg + k) % 3;
        const int e = ie[(d0 + k) % 3];
        if (symstart[ax] == 0.0 || e <= symstart[ax]) {
            is[k] = e;
        } else {
            const int a = (int)fabs(2.0 * symstart[ax] - e);
            is[k] = a > 1 ? a : 1;
        }
    }
}

/* ---------------------------------------------------------------- topologies */
/* src/flups.h:210 */
FLUPS_Topology* flups_topo_new(const int axis, const int lda, const int nglob[3], const int nproc[3], const bool isComplex,
                               const int axproc[3], const int alignment, MPI_Comm comm);
/* src/flups.h:217 */
void flups_topo_free(const FLUPS_Topology* t);
/* src/flups.h:226 */
bool flups_topo_get_isComplex(const FLUPS_Topology* t);
/* src/flups.h:234 */
int flups_topo_get_lda(const FLUPS_Topology* t);
/* src/flups.h:242 */
int flups_topo_get_axis(const FLUPS_Topology* t);
/* src/flups.h:250 */
int flups_topo_get_nglob(const FLUPS_Topology* t, const int dim);
/* src/flups.h:261 */
int flups_topo_get_nloc(const FLUPS_Topology* t, const int dim);
/* src/flups.h:272 */
int flups_topo_get_nmem(const FLUPS_Topology* t, const int dim);
/* src/flups.h:280 */
int flups_topo_get_nproc(const FLUPS_Topology* t, const int dim);
/* src/flups.h:287 */
void flups_topo_get_istartGlob(const FLUPS_Topology* t, int istart[3]);
/* src/flups.h:294 */
size_t flups_topo_get_locsize(const FLUPS_Topology* t);
/* src/flups.h:301 */
size_t flups_topo_get_memsize(const FLUPS_Topology* t);
/* src/flups.h:314 */
int flups_topo_cmpt_rank_fromid(const FLUPS_Topology* t, const int global_id, const int id);
/* src/flups.h:321 */
int flups_topo_cmpt_start_id_from_rank(const FLUPS_Topology* t, const int rank_id, const int id);
/* src/flups.h:329 */
MPI_Comm flups_topo_get_comm(FLUPS_Topology* t);
/* src/flups.h:340 */
void flups_topo_ranksplit(const FLUPS_Topology* t, const int rank, int rankd[3]);
/* src/flups.h:349 */
int flups_topo_rankindex(const FLUPS_Topology* topo, const int rankd[3]);

/* ---------------------------------------------------------------- solver */
/* src/flups.h:369 */
FLUPS_Solver* flups_init(FLUPS_Topology* t, FLUPS_BoundaryType* bc[3][2], const double h[3], const double L[3],
                         FLUPS_DiffType orderDiff, const FLUPS_CenterType center_type[3]);
/* src/flups.h:375 */
FLUPS_Solver* flups_init_timed(FLUPS_Topology* t, FLUPS_BoundaryType* bc[3][2], const double h[3], const double L[3],
                               const FLUPS_DiffType orderDiff, const FLUPS_CenterType center_type[3], FLUPS_Profiler* prof);
/* src/flups.h:384 */
void flups_cleanup(FLUPS_Solver* s);
/* src/flups.h:392 */
void flups_cleanup_solver(FLUPS_Solver* s);
/* src/flups.h:401 */
void flups_cleanup_all(FLUPS_Solver* s);
/* src/flups.h:410 */
void flups_cleanup_backend(void);
/* src/flups.h:421 */
void flups_set_greenType(FLUPS_Solver* s, const FLUPS_GreenType type);
/* src/flups.h:429 -- stream is a cudaStream_t */
void flups_set_stream(FLUPS_Solver* s, void* stream);
/* src/flups.h:441 */
void flups_setup(FLUPS_Solver* s, const bool changeComm);
/* src/flups.h:452 -- field and rhs may alias; host or device pointers */
void flups_solve(FLUPS_Solver* s, double* field, double* rhs, const FLUPS_SolverType type);

/* ---------------------------------------------------------------- advanced */
/* src/flups.h:473 */
size_t flups_get_allocSize(FLUPS_Solver* s);
/* src/flups.h:485 */
void flups_get_spectralInfo(FLUPS_Solver* s, double kfact[3], double koffset[3], double symstart[3]);
/* src/flups.h:494 */
void flups_set_alpha(FLUPS_Solver* s, const double alpha);
/* src/flups.h:509 -- the solver's inner buffer: managed memory (host and
 * device), doubles, large enough for both inner layouts */
double* flups_get_innerBuffer(FLUPS_Solver* s);
/* src/flups.h:517 -- owned by the solver: the user layout (there are no pencils) */
FLUPS_Topology* flups_get_innerTopo_physical(FLUPS_Solver* s);
/* src/flups.h:525 -- owned by the solver: the full spectrum, axis 0, nf = 2 */
FLUPS_Topology* flups_get_innerTopo_spectral(FLUPS_Solver* s);
/* src/flups.h:534 -- accepted, no effect: the physical inner layout is the user's */
void flups_skip_firstSwitchtopo(FLUPS_Solver* s);
/* src/flups.h:544 -- host or device data in the physical topology <-> inner buffer */
void flups_do_copy(FLUPS_Solver* s, const FLUPS_Topology* topo, double* data, const int sign);
/* src/flups.h:552 -- data is the inner buffer: FLUPS_FORWARD from the physical
 * to the spectral layout, FLUPS_BACKWARD (or FLUPS_BACKWARD_DIFF after a ROT
 * multiply) back; the unnormalised transforms of the reference */
void flups_do_FFT(FLUPS_Solver* s, double* data, const int sign);
/* src/flups.h:560 -- normfact * Green (STD) or normfact * Green * curl (ROT) */
void flups_do_mult(FLUPS_Solver* s, double* data, const FLUPS_SolverType type);
/* src/flups.h:570 */
void flups_pencilDirs(const FLUPS_BoundaryType* bc[3][2], int dirs[3]);
/* src/flups.h:578 */
void flups_switchtopo_info(FLUPS_Solver* s);

/* ---------------------------------------------------------------- profiler */
/* src/flups.h:592-611 -- named wall-clock/CUDA-event timers */
FLUPS_Profiler* flups_profiler_new(void);
FLUPS_Profiler* flups_profiler_new_n(const char name[]);
void flups_profiler_free(FLUPS_Profiler* p);
void flups_profiler_disp(FLUPS_Profiler* p);

/* ---------------------------------------------------------------- output */
/* src/flups.h:634 -- writes <filename>.bin raw doubles and a .xmf description into ./data */
void flups_hdf5_dump(const FLUPS_Topology* topo, const char filename[], const double* data);
/* src/flups.h:638 */
void flups_print_data(const FLUPS_Topology* topo, double* data);

#ifdef __cplusplus
}
#endif

#include "flups_b200.h"

#endif
