// Host-side layout, plan tables and solver of the B200 FLUPS library.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "../../include/flups.h"
#include "fast_dft.h"
#include "green.cuh"
#include "pass_desc.h"

#define FLB_CHECK(cond, ...)                                                        \
    do {                                                                            \
        if (!(cond)) {                                                              \
            fprintf(stderr, "[flups_b200] error in %s: ", __func__);               \
            fprintf(stderr, __VA_ARGS__);                                           \
            fprintf(stderr, "\n");                                                  \
            fflush(stderr);                                                         \
            abort();                                                                \
        }                                                                           \
    } while (0)

namespace flb {

cudaError_t launch_line_pass(const PassArgs& A, int compute_f64, int in_f64, int out_f64, cudaStream_t stream);
size_t line_pass_smem(const PassArgs& A, int elem_bytes);
cudaError_t launch_green_eval(const GreenEvalArgs& A, cudaStream_t s);
cudaError_t launch_green_final(const GreenFinalArgs& A, cudaStream_t s);

// plan types and FFTW r2r kinds (src/FFTW_plan_dim.hpp:34-62)
enum PlanType { SYMSYM = 2, MIXUNB = 5, PERPER = 6, UNBUNB = 8, EMPTY = 18 };
enum R2RKind { K_NONE = 0, REDFT00, REDFT10, REDFT01, REDFT11, RODFT00, RODFT10, RODFT01, RODFT11 };

// One direction's transform: a restatement of the tables of FFTW_plan_dim
// (src/FFTW_plan_dim.cpp:77-161) and of its cell/node initialisers
// (src/FFTW_plan_dim_cell.cpp:19-390, src/FFTW_plan_dim_node.cpp:19-461).
struct DirPlan {
    int lda = 1, dim = 0, sign = FLUPS_FORWARD;
    bool is_green = false;
    int center = CELL_CENTER;
    int bc[2][3] = {{0, 0, 0}, {0, 0, 0}};
    int type = EMPTY;
    double volfact = 1.0, kfact = 0.0, normfact = 1.0, symstart = 0.0, koffset = 0.0;
    bool is_spectral = false, isr2c = false;
    int n_in[3] = {1, 1, 1}, fstart_in[3] = {0, 0, 0}, fstart_out[3] = {0, 0, 0}, postpro[3] = {0, 0, 0};
    bool imult[3] = {false, false, false};
    int kind[3] = {K_NONE, K_NONE, K_NONE};
    int n_out = 1, fieldstart = 0;

    DirPlan() = default;
    DirPlan(int lda, int dim, const double h[3], const double L[3], const int bcl[3], const int bcr[3], int sign, bool green,
            int center);
    bool isr2c_done_by_fft() const { return isr2c && !is_spectral; }
    void init(const int size[3], bool is_complex);

   private:
    void r2r_cell(int n);
    void mix_cell(int n);
    void per_cell(int n, bool c);
    void unb_cell(int n, bool c);
    void r2r_node(int n);
    void mix_node(int n);
    void per_node(int n, bool c);
    void unb_node(int n, bool c);
};

void sort_plans(DirPlan p[3]);

}  // namespace flb

struct Solver;
namespace flb {
// drops the group graphs (flups_b200_solve_group) that hold a solver being destroyed
void group_forget(const Solver* s);
}  // namespace flb

// Opaque handles of the C API
struct Topology {
    int axis = 0, lda = 1, nf = 1, alignment = FLUPS_ALIGNMENT;
    int nglob[3] = {1, 1, 1}, nloc[3] = {1, 1, 1}, nmem[3] = {1, 1, 1}, nproc[3] = {1, 1, 1}, axproc[3] = {0, 1, 2};
    MPI_Comm comm = 0;
    void cmpt_sizes();  // src/Topology.cpp:81-98
    size_t memdim() const { return (size_t)nmem[0] * nmem[1] * nmem[2] * nf; }
    size_t memsize() const { return memdim() * lda; }
    size_t locsize() const { return (size_t)nloc[0] * nloc[1] * nloc[2] * nf; }
};

struct Profiler {
    std::string name;
    std::map<std::string, double> acc_ms;
    std::map<std::string, long> count;
};

// Array state between passes: extents along x, y, z and element type.
struct ArrState {
    int n[3];
    bool cplx;
};

struct Solver {
    // ---------------------------------------------------------------- inputs
    Topology* topo_phys = nullptr;
    int lda = 1;
    double h[3] = {1, 1, 1}, L[3] = {1, 1, 1};
    int odiff = NOD;
    int center = CELL_CENTER;
    int bc[3][2][3];
    int green_type = CHAT_2;
    double alpha = 2.0;
    int precision = 64;
    bool async = false;
    bool skip_st0 = false;
    cudaStream_t stream = 0;
    Profiler* prof = nullptr;
    int last_error = 0;
    // ---------------------------------------------------------------- plans
    flb::DirPlan fwd[3], bwd[3], grn[3], dif[3];
    bool have_diff = false;
    int ndim = 3;
    double normfact = 1.0, volfact = 1.0;
    ArrState st[4];            // st[k]: array after k forward transforms
    int sizes_before[3][3];    // size before forward plan ip
    // ---------------------------------------------------------------- device data
    bool is_setup = false;
    void* buf[2] = {nullptr, nullptr};    // work arrays (working precision)
    size_t buf_elems[2] = {0, 0};         // capacity in reals
    int buf_batch = 0;
    void* green = nullptr;                // folded Green's spectrum (working precision)
    int gfold_M[3] = {0, 0, 0}, gfold_n[3] = {1, 1, 1};
    int64_t gstr[3] = {1, 1, 1};
    std::map<int64_t, void*> twiddles;    // key: M * 2 + (precision == 64)
    double* stage_in = nullptr;           // device staging for host rhs/field
    size_t stage_elems = 0;
    // host-array solves: copies in slabs along the last forward direction,
    // overlapped with the passes of the other slabs (and, with async, with the
    // copies of the previous and next solve)
    static constexpr int kSlabs = 8;
    double* stage_out = nullptr;          // device staging for a host field (separate from stage_in)
    size_t stage_out_elems = 0;
    cudaStream_t h2d_stream = nullptr, d2h_stream = nullptr;
    cudaEvent_t ev_in[kSlabs] = {}, ev_fwd[kSlabs] = {}, ev_bwd[kSlabs] = {}, ev_out[kSlabs] = {};
    // async host-array solves run their passes on cstream: the caller's
    // stream waits for each solve's last download, and the next such solve
    // need not (cs_follows: the solver's last work was such a solve, so its
    // passes are ordered behind the previous ones on cstream already)
    cudaStream_t cstream = nullptr;
    cudaEvent_t ev_entry = nullptr;
    bool cs_follows = false;
    // host range [dl_lo, dl_hi) that the last streamed download writes (its
    // slabs finish at ev_out): a later upload reading it waits for them
    const char* dl_lo = nullptr;
    const char* dl_hi = nullptr;
    int slab_dim = -1, slab_lo = 0, slab_hi = 0;   // restriction run_pass applies to non-fused passes
    double* inner = nullptr;              // spectral buffer of the advanced API (doubles)
    Topology* topo_spec = nullptr;
    Topology* topo_inner_phys = nullptr;
    // ---------------------------------------------------------------- host-only planning
    bool dry = false;                     // record passes instead of launching them
    std::vector<flb::PassArgs> dry_passes;
    std::vector<int> dry_flags;
    std::vector<std::string> dry_names;
    std::vector<int> dry_fast;
    bool use_fast = true;                 // register-resident power-of-two kernels where they apply
    // ---------------------------------------------------------------- per-pass timing
    bool timing = false;
    int pass_idx = 0;
    // CTA-tile autotuning of the column passes: per pass signature, the tile
    // that ran fastest on this GPU (timed once per signature, before the solve)
    bool autotune = false;
    int force_tile = 0;                     // COL_TILE_* for every column pass (0: default / tuned)
    std::map<std::string, int> tuned_tile;
    std::map<int64_t, bool> tuned_solves;   // (type, nbatch) already tuned
    // solves captured in CUDA graphs, keyed by (field, rhs, nbatch, type)
    struct GraphKey {
        const void* field;
        const void* rhs;
        int nbatch, type;
        bool operator<(const GraphKey& o) const {
            if (field != o.field) return field < o.field;
            if (rhs != o.rhs) return rhs < o.rhs;
            if (nbatch != o.nbatch) return nbatch < o.nbatch;
            return type < o.type;
        }
    };
    std::map<GraphKey, cudaGraphExec_t> graphs;
    cudaStream_t capture_stream = nullptr;
    bool capturing = false;
    uint64_t gen = 0;                     // bumped whenever captured solves become stale
    void drop_graphs();
    std::string pass_key(const flb::PassArgs& A, bool f64) const;
    void autotune_passes(int type, int nbatch);
    int solve_graph(double* field, double* rhs, int type, int nbatch);
    std::vector<cudaEvent_t> ev;          // 2 per pass of the last solve
    std::vector<double> pass_ms, pass_bytes;
    std::vector<long> pass_calls;
    std::vector<std::string> pass_names;

    Solver(Topology* t, FLUPS_BoundaryType* bc[3][2], const double h[3], const double L[3], int odiff, const int center[3],
           Profiler* prof);
    ~Solver();
    void setup();
    void solve(double* field, double* rhs, int type, int nbatch);
    size_t alloc_size() const;
    size_t device_bytes(int nbatch) const;
    void spectral_info(double kfact[3], double koffset[3], double symstart[3]) const;

    // ---------------------------------------------------------------- internals
    void dry_run(flb::DirPlan p[3]);
    void compute_green();
    const void* twiddle(int M, bool f64);
    const void* twiddle_plain(int L, bool f64);   // W_L^q, q < L
    // later-stage twiddles of an n-point register DFT with first radix r1 (0: the default of the precision)
    const void* stage_table(int n, bool f64, int r1 = 0);
    // 0 none, 1 column c2c, 2 row r2c/c2r, 3 column r2c/c2r, 4 row r2r, 5 fused row
    int fast_kind(const flb::PassArgs& A, bool f64, bool in_f64, bool out_f64) const;
    // arguments of a fast launch, all but the twiddle tables; mode of a column pass
    void fast_args(const flb::PassArgs& A, int kind, bool in_f64, bool out_f64, flb::ColArgs& c, flb::RowArgs& r, int& mode) const;
    void launch_fast(const flb::PassArgs& A, int kind, bool f64, bool in_f64, bool out_f64);
    void rowfused_args(const flb::PassArgs& A, flb::RowFusedArgs& f) const;
    void ensure_buffers(int nbatch);
    flb::LineStage stage_forward(const flb::DirPlan& p, int ip, bool f64);
    flb::LineStage stage_backward(const flb::DirPlan& p, const flb::DirPlan& pf, int ip, bool f64);
    flb::PassArgs base_pass(int axis, const ArrState& src, int ncomp, int lda_spec);
    void set_strides_internal(int64_t str[3], int64_t& cstr, const ArrState& s, bool pad = true) const;
    int64_t row_pitch(const ArrState& s) const;             // x extent in memory (128-byte multiple)
    size_t state_reals(int k, int nbatch) const;            // reals held by state k for nbatch right-hand sides
    size_t work_reals(int b, int nbatch) const;             // reals of work array b (both pass orders)
    void set_strides_user(int64_t str[3], int64_t& cstr) const;
    void fit_lines(flb::PassArgs& A, int elem_bytes) const;
    flb::MultSpec mult_spec(int type) const;
    void run_pass(const flb::PassArgs& A, bool f64, bool in_f64, bool out_f64, const char* name = "pass");
    int timed_begin(const char* name, double bytes);
    void timed_end(int k);
    // ---------------------------------------------------------------- advanced API (flups.h:473-578)
    size_t inner_elems = 0;               // doubles in the inner buffer
    int64_t inner_pitch = 0;              // complex row pitch of the spectral layout
    void ensure_inner();
    void inner_spec_strides(int64_t str[3], int64_t& cstr) const;
    void adv_copy(const Topology* topo, double* data, int sign);
    void adv_fft(double* data, int sign);
    void adv_mult(double* data, int type);
    // curl symbols of the fused ROT pass: K_{d,c}(i) per direction d and
    // component c, kstr complex values each (working precision), built at set-up
    void* ksym = nullptr;
    int kstr = 0;
    void build_ksym();
    // x-last order of an all-unbounded 3-D problem: z (r2c), y, x, so that the
    // last direction (forward DFT, multiply, inverse DFT) runs along
    // contiguous rows, one warp per row.  Solves of device arrays use it; the
    // reference's order (fwd/bwd/grn/dif) stays the public one (plan tables,
    // advanced API, host-array and z-slab solves).  swap_order() exchanges
    // the two sets for the duration of a solve; the folded Green's spectrum
    // is the same array in both orders.
    bool has_xlast = false;
    bool xlast_mixed = false;  // the x-last plans include a periodic direction
    bool xlast_on = true;                 // flups_b200_set_xlast
    bool xlast_active = false;
    flb::DirPlan xfwd[3], xbwd[3], xdif[3];
    ArrState xst[4];
    int xgfold_M[3] = {0, 0, 0};
    void* xksym = nullptr;
    int xkstr = 0;
    bool xlast_fast[2] = {false, false};  // STD, ROT: every pass of the x-last order is a register-DFT kernel
    void build_xlast();
    void swap_order();
    void plan_xlast();
    bool xlast_ok(int type) const;
    void collect_timing();
    void check_cuda(cudaError_t e, const char* what);
    void do_fft_forward(const double* user_in, int nbatch);
    void fwd_pass(int ip, const double* user_in, int nbatch);
    void bwd_pass(int ip, double* user_out, int type, int nbatch);
    // overlapped middle passes over x-slabs (flups_b200_set_overlap)
    bool overlap = false;
    // L2 prefetch of the next blocks' input in the row and column passes (flups_b200_set_prefetch)
    bool prefetch = true;
    void col_prefetch(flb::ColArgs& c, bool f64, int L, int ncomp) const;
    void row_prefetch(flb::RowArgs& r, bool f64, bool c2r, int L, int ncomp) const;
    void rowrot_prefetch(flb::RowFusedArgs& f, bool f64, int L, int ncomp) const;
    static constexpr int kOvSlabs = 4;
    cudaStream_t ov_stream[2] = {nullptr, nullptr};
    cudaEvent_t ov_ev0 = nullptr, ov_evf[kOvSlabs] = {}, ov_evg[kOvSlabs] = {};
    bool overlap_ok(int type) const;
    void solve_overlap(const double* din, double* dout, int type, int nbatch);
    void do_fused(int type, int nbatch);
    void do_backward(double* user_out, int type, int nbatch);
    void do_fft_backward_fused(double* user_out, int type, int nbatch);
    bool streamed_ok() const;
    void solve_streamed(double* field, double* rhs, bool in_host, bool out_host, int type, int nbatch, bool follows);
    void restrict_slab(flb::PassArgs& A, bool in_f64, bool out_f64) const;
    // one rank's steps of a z-slab decomposed solve (flups_b200_slab_*): the
    // x and y passes of user planes [z0, z1), the last-direction pass of
    // spectrum columns [x0, x1) over every plane, the inverse x and y passes
    // of planes [z0, z1); the caller moves the spectrum between ranks
    // ownership set before setup (flups_b200_slab_own): planes [own[0], own[1])
    // and spectrum columns [own[2], own[3]); the work arrays then hold those
    // planes only, and `xbuf` (pitch `xpitch`) holds the columns over every plane
    int own[4] = {-1, -1, -1, -1};
    void* xbuf = nullptr;
    int64_t xpitch = 0;
    bool owned() const { return own[0] >= 0; }
    int slab_own(int z0, int z1, int x0, int x1);
    void* green_share = nullptr;  // allocation of a share's columns of the Green's spectrum
    // every rank's column array (flups_b200_slab_peers): the y passes of a
    // share write / read them directly instead of the plane array
    flb::ColArgs::Peers peers{};
    int slab_peers(int n, void* const* cols, const int* xs, const int64_t* pitch);
    bool slab_y_fast();
    void slice_green();
    void* work_base(int b) const;
    int slab_check(int type) const;
    int slab_forward(const double* rhs);
    int slab_fused(int type);
    int slab_backward(double* field, int type);
    std::string plan_json(int type, int nbatch);
};
