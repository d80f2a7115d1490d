/*
 * flups_b200.h -- entry points added by the B200 library.  None changes the
 * meaning of a reference call: a caller that never uses them gets the
 * reference's behaviour (FP64 arithmetic, synchronous flups_solve).
 */
#ifndef FLUPS_B200_H
#define FLUPS_B200_H

#include <stddef.h>
#include <stdint.h>

#include "flups_mpi.h"

#ifdef __cplusplus
extern "C" {
#else
#include <stdbool.h>
#endif

struct Solver;
struct Topology;

/* Arithmetic of the per-solve transforms: 64 (default, as the reference) or
 * 32 (FP32 transforms with FP64-computed twiddles and an FP32 copy of the
 * FP64 Green's spectrum).  Must be called before flups_setup.  No reference
 * counterpart (the reference is FP64 only, src/Solver.hpp:67,102). */
void flups_set_precision(struct Solver* s, int bits);
int flups_get_precision(struct Solver* s);

/* Solve nbatch independent right-hand sides sharing one Green's spectrum in
 * one sequence of launches.  rhs and field hold nbatch consecutive arrays of
 * flups_topo_get_memsize(topo) doubles each (host or device pointers).  No
 * reference counterpart; equivalent to nbatch calls of flups_solve. */
void flups_solve_batch(struct Solver* s, double* field, double* rhs, int nbatch, int type);

/* When set, flups_solve returns once its work is queued on the solver's
 * stream, without synchronising.  With host arrays the upload of rhs and the
 * download of field run on the library's copy streams in slabs, overlapped
 * with the transforms and with the copies of the previous and next solve;
 * rhs and field must stay untouched until the solve is complete (for host
 * arrays page-locked memory lets the copies run asynchronously), and a host
 * rhs must hold its values when the call is made (its upload does not wait
 * for other work on the stream; it does wait for an earlier solve's download
 * into the same memory, so chained and in-place calls are safe).  Solves of
 * host arrays in and out run their transforms on a library stream, so one
 * solve's download overlaps the next one's transforms.  Completion is
 * ordered before later work on the solver's stream; flups_synchronize waits
 * for it.  Default 0 (every call returns with its result in place). */
void flups_set_async(struct Solver* s, int async);

/* Wait for every solve queued on the solver's stream (async mode). */
void flups_synchronize(struct Solver* s);

/* Last CUDA error seen by the solver (0 = none).  No reference counterpart:
 * the reference aborts on every error (src/defines.hpp:301-304). */
int flups_get_last_error(struct Solver* s);

/* Device bytes the solver holds after flups_setup (work buffers, Green's
 * spectrum, twiddle tables) for nbatch right-hand sides. */
size_t flups_get_device_bytes(struct Solver* s, int nbatch);

/* Per-pass device timing of the following solves (CUDA events around each
 * line pass on the solver's stream), for profiling; on = 0 stops recording
 * and both calls reset the counters.  flups_get_pass_stats returns the number
 * of passes per solve and fills, per pass, the accumulated milliseconds, the
 * algorithmic bytes of one launch (source and kept output read/written once,
 * the folded Green's spectrum once), the number of timed launches and a name
 * (name_len bytes each).  Plays the part of the reference's profiler labels
 * "fftw"/"SwitchTopo"/"domagic" (src/Solver.cpp:1411-1475). */
void flups_set_pass_timing(struct Solver* s, int on);
int flups_get_pass_stats(struct Solver* s, int maxn, double* ms_total, double* bytes, long* calls, char* names, int name_len);

/* Host-only description (JSON) of the solver's per-direction tables and of
 * the line passes one solve of kind type over nbatch right-hand sides would
 * launch; needs no GPU.  Returns the length needed including the final NUL
 * (the output is truncated to len).  For tests and tooling. */
int flups_b200_plan_json(struct Solver* s, int type, int nbatch, char* out, int len);

/* Use (1, default) or bypass (0) the register-resident power-of-two DFT
 * kernels; with 0 every pass runs through the general line-pass kernel.
 * For cross-checking the two kernel families. */
void flups_b200_set_fast_kernels(struct Solver* s, int on);

/* CTA-tile autotuning of the column passes (1 = on, default 0).  When on,
 * the first solve of each (solver type, nbatch) times the two compiled tiles
 * of every column pass on the solver's work arrays and keeps the faster one;
 * that first call synchronises the stream.  No reference counterpart. */
void flups_b200_set_autotune(struct Solver* s, int on);

/* Overlap the middle passes of a solve of device arrays (1 = on, default 0):
 * after the x transform, the y forward, fused z and y inverse passes run per
 * x-slab on three streams, so one slab's fused pass (bound by arithmetic)
 * runs beside other slabs' y passes (bound by memory).  Results are
 * identical.  No reference counterpart. */
void flups_b200_set_overlap(struct Solver* s, int on);

/* L2 prefetch in the register-DFT row passes and the forward / inverse
 * column passes (1 = on, the default): each CTA asks the TMA unit to bring
 * the input of the CTA launched 148 blocks later into L2, so that CTA's
 * loads hit L2.  Results are identical either way.  No reference
 * counterpart. */
void flups_b200_set_prefetch(struct Solver* s, int on);

/* Pass order of 3-D solves of device arrays whose directions are all
 * unbounded or periodic (ROT: when x is the reference's first direction)
 * (1 = x last, the default; 0 = the reference's order).  With x last, z is the
 * real-to-complex direction and the last pass -- forward DFT, Green's
 * multiply, inverse DFT -- runs along contiguous x rows, one warp per row
 * (1.28 against 2.04 ms for that pass at 512^3 FP32).  The result equals the
 * other order's to rounding.  Host-array (streamed) solves, the advanced API
 * and z-slab solves keep the reference's order.  No reference counterpart. */
void flups_b200_set_xlast(struct Solver* s, int on);

/* Force the CTA tile of every column pass: 0 = default or tuned, 1 = 256
 * threads, 2 = 128 threads.  For cross-checking the tiles. */
void flups_b200_set_col_tile(struct Solver* s, int tile);

/* One rank's share of a solve split over ranks by planes of the last
 * direction; replaces the reference's multi-rank pencil solve
 * (src/Solver.cpp:629-715 with src/SwitchTopoX_a2a.cpp:118-247), whose
 * transposes become two all-to-all exchanges of the spectrum that the
 * caller does (flups_b200/slab.py: torch.distributed / NCCL).  Rank r owns
 * user planes [z0, z1) and spectrum columns [x0, x1); scalar fields, STD,
 * directions x, y, z transformed in that order (else -2; -1: wrong order of
 * calls).  A rank's work arrays hold its planes and its columns only, and
 * set-up keeps only its columns of the Green's spectrum.
 *   flups_b200_slab_info: spectrum extents (info[0..2] = nx, ny, nz), row
 *     pitch of the plane array in complex values (info[3]), user planes
 *     (info[4]), row pitch of the column array (info[5], after slab_own),
 *     bytes per real (info[6]); returns 0 when the problem qualifies.
 *   flups_b200_slab_own: before flups_setup, the planes and columns this
 *     solver owns (flups_solve and the advanced calls then refuse it).
 *   flups_b200_slab_planes: device array of the owned planes of the spectrum
 *     between the passes, complex value (x, y, z - z0) at
 *     x + pitch (y + ny (z - z0)).
 *   flups_b200_slab_columns: device array of the owned columns over every
 *     plane, complex value (x - x0, y, z) at (x - x0) + cpitch (y + ny z).
 *   flups_b200_slab_forward: x and y forward passes of the owned planes of
 *     rhs (device array holding those planes only, user layout) into the
 *     plane array.
 *   flups_b200_slab_fused: last-direction pass (forward DFT, Green's
 *     multiply, inverse DFT) of the column array, in place.
 *   flups_b200_slab_backward: y and x inverse passes of the plane array into
 *     field (the owned planes only).
 * Between forward and fused the caller moves block (owned planes, columns of
 * rank j) of every rank's plane array into rank j's column array, and back
 * between fused and backward.  Each step is the single-rank pass restricted
 * to a slab: the assembled field equals flups_solve's bit for bit. */
int flups_b200_slab_info(struct Solver* s, int64_t info[7]);
int flups_b200_slab_own(struct Solver* s, int z0, int z1, int x0, int x1);
void* flups_b200_slab_planes(struct Solver* s);
void* flups_b200_slab_columns(struct Solver* s);
int flups_b200_slab_forward(struct Solver* s, const double* rhs);
int flups_b200_slab_fused(struct Solver* s, int type);
int flups_b200_slab_backward(struct Solver* s, double* field, int type);
/* The column arrays of every rank (n ranks, n <= 8; rank j owns columns
 * [xs[j], xs[j+1]) with row pitch pitch[j]; this solver's own entry is its
 * flups_b200_slab_columns array): the y forward pass of flups_b200_slab_forward
 * then stores each column straight into its owner's array and the y inverse
 * pass of flups_b200_slab_backward loads it from there, over NVLink for the
 * arrays of other GPUs (opened with flups_b200_ipc_open), so no exchange
 * copies remain; the caller only orders the steps across ranks (every
 * rank's forward before any fused step, every fused step before any
 * backward, every backward before the next forward).  n = 0 returns to the
 * plane array.  Returns 0, -1 (not a set-up share) or -2 (bad table). */
int flups_b200_slab_peers(struct Solver* s, int n, void* const* cols, const int* xs, const int64_t* pitch);
/* CUDA IPC of a device allocation (cudaIpcGetMemHandle /
 * cudaIpcOpenMemHandle with lazy peer access / cudaIpcCloseMemHandle); the
 * handle is 64 bytes.  Return 0, -2 (bad arguments) or -4 (CUDA error). */
int flups_b200_ipc_handle(const void* dev_ptr, void* handle);
int flups_b200_ipc_open(const void* handle, void** dev_ptr);
int flups_b200_ipc_close(void* dev_ptr);

/* A solve (nbatch consecutive right-hand sides, as flups_solve_batch) of
 * device arrays replayed from a CUDA graph.  The first call for a given
 * (field, rhs, nbatch, type) runs one plain solve, then captures the next
 * into a graph; later calls only launch the graph on the solver's stream.
 * Graphs are dropped when the solver reallocates its work arrays and at
 * cleanup.  Synchronises unless flups_set_async(s, 1).  Returns 0, -1 (not
 * set up or bad arguments), -2 (host pointers) or -4 (CUDA error, also in
 * flups_get_last_error).  No reference counterpart (the reference launches
 * FFTW plans, src/Solver.cpp:1207-1272). */
int flups_solve_graph(struct Solver* s, double* field, double* rhs, int nbatch, int type);

/* Solves of n different solvers -- unevenly sized grids, other boundary
 * conditions, kernels, precisions or solver types (STD / ROT) -- as ONE CUDA
 * graph launched on `stream` (a cudaStream_t; NULL = the default stream).
 * fields[i] and rhss[i] are device arrays of solver ss[i] (set up, not a
 * z-slab share); a solver appears once (its work arrays are one set).  The
 * first call for a given (solvers, arrays, types) runs each solve once,
 * then captures them as independent branches of one graph, so the small
 * grids' passes run side by side; later calls launch that graph (a member
 * whose work arrays grew or whose switches changed gets the group
 * recaptured; destroying a member drops its groups).  The call returns once
 * the graph is queued: synchronise `stream` before reading the fields.
 * Returns 0, -1 (bad arguments or a solver not set up), -2 (host pointers,
 * a solver or an output twice) or -4 (CUDA error, in flups_get_last_error
 * of every member).  No reference counterpart (the reference solves one
 * field per call). */
int flups_b200_solve_group(struct Solver* const* ss, int n, double* const* fields, double* const* rhss, const int* types,
                           void* stream);

/* One solve that allocates no device memory, for callers that cannot call
 * cudaMalloc while they run: real-time loops that must stay out of the
 * allocator (cudaMalloc can synchronise the device and takes driver locks,
 * so its latency has no bound), and frameworks that reserve the device
 * memory for their own pools at start-up, after which a cudaMalloc fails.
 * No counterpart in the reference (its solve allocates nothing per call but
 * runs on the host).  The per-solve scratch (work arrays and twiddle tables)
 * lives in one file-scope device array of 64 MiB held by every GPU that
 * loads the library until the process exits; solves that need more are
 * refused (return -3).  field and rhs must be device pointers, flups_setup
 * must have run (it allocates), and the call only enqueues on the solver's
 * stream (synchronise before reading field).  The first call on a device
 * looks up the array's address (cudaGetSymbolAddress): make it before any
 * stream capture.  All calls share the array and it keeps the last call's
 * contents, so calls that may overlap on the GPU race; nothing in it has to
 * start at zero.  Returns 0, or a negative code with a message on stderr
 * (-1 not set up, -2 bad arguments, -3 too large, -4 CUDA error). */
int flups_solve_noalloc(struct Solver* s, double* field, double* rhs, int type);

/* Alternative names of two reference calls:
 * flups_init_topology == flups_topo_new (src/flups.h:210) and
 * flups_solve_rot == flups_solve(..., ROT) (src/flups.h:452). */
struct Topology* flups_init_topology(const int axis, const int lda, const int nglob[3], const int nproc[3], const bool isComplex,
                                     const int axproc[3], const int alignment, MPI_Comm comm);
void flups_solve_rot(struct Solver* s, double* field, double* rhs);

#ifdef __cplusplus
}
#endif

#endif
