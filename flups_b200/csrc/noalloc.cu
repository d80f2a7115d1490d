// flups_solve_noalloc: a solve that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they run: real-time loops that
// must stay out of the allocator (cudaMalloc can synchronise the device and
// takes driver locks, so its latency has no bound), and frameworks that
// reserve the device memory for their own pools at start-up, after which a
// late cudaMalloc fails.  For them this entry point runs one solve of an
// already set-up solver with all of its per-solve scratch -- the two work
// arrays between the line passes and the twiddle tables of those passes -- in
// one file-scope device array of FLUPS_NOALLOC_SCRATCH_BYTES (64 MiB).  Every
// GPU that loads the library holds that array until the process exits.
//
// Rules for callers:
//   - field and rhs must be device pointers: there is no host staging;
//   - flups_setup must have run: the Green's spectrum it computes is an input
//     here (setup allocates; this call does not);
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress; make that first call before any stream capture;
//   - the call only enqueues work on the solver's stream (flups_set_stream)
//     and returns; synchronise that stream before reading field;
//   - every call shares the array and overwrites what the previous call left
//     in it: calls that may overlap on the GPU (different streams without an
//     ordering between them) race on it;
//   - nothing in the array has to start at zero (the passes write every
//     element they later read; the twiddle tables are rewritten per call);
//   - a solve whose scratch does not fit is refused with an error code.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "fast_dft.h"
#include "host.hpp"

#define FLUPS_NOALLOC_SCRATCH_BYTES (64u << 20)
#define FLUPS_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[FLUPS_NOALLOC_SCRATCH_BYTES];
static void* g_noalloc_ptr[FLUPS_NOALLOC_MAX_DEVICES] = {nullptr};

using namespace flb;

// exp(-2 pi i q / n) for q < n (stage == 0), or the later-stage table of an
// n-point register DFT (stage == 1); FP64 sincospi, stored in the working precision
__global__ void noalloc_twiddle_kernel(void* out, int n, int stage, int len, int r1, int f64) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < len; e += gridDim.x * blockDim.x) {
        int q = e, M = n;
        if (stage) fast_stage_exponent(n, r1, e, &q, &M);
        double s, c;
        sincospi(-2.0 * (double)q / (double)M, &s, &c);
        if (f64) reinterpret_cast<double2*>(out)[e] = make_double2(c, s);
        else reinterpret_cast<float2*>(out)[e] = make_float2((float)c, (float)s);
    }
}

namespace {

struct TwSlot {
    int n;        // transform length
    int stage;    // 0: W_n^q table; r1 > 0: later-stage table of an n-point register DFT of first radix r1
    int len;      // complex entries
    size_t off;   // byte offset in the scratch array
};

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

int fail(int code, const char* msg) {
    fprintf(stderr, "[flups_b200] flups_solve_noalloc: %s\n", msg);
    fflush(stderr);
    return code;
}

}  // namespace

extern "C" int flups_solve_noalloc(Solver* s, double* field, double* rhs, int type) {
    if (!s) return fail(-1, "solver is NULL");
    if (!s->is_setup) return fail(-1, "flups_setup must be called first (it computes the Green's spectrum)");
    if (s->owned()) return fail(-2, "this solver holds one rank's share of the planes (flups_b200_slab_own)");
    if (!field || !rhs) return fail(-2, "field and rhs must not be NULL");
    if (type == ROT && (s->lda != 3 || s->odiff == NOD)) return fail(-2, "ROT needs lda = 3 and a derivative order");
    for (const void* p : {(const void*)field, (const void*)rhs}) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess ||
            !(a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged)) {
            cudaGetLastError();
            return fail(-2, "field and rhs must be device pointers (no host staging without allocation)");
        }
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= FLUPS_NOALLOC_MAX_DEVICES) return fail(-4, "no usable device");
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            s->last_error = (int)e;
            return fail(-4, "cudaGetSymbolAddress of the scratch array failed");
        }
        g_noalloc_ptr[dev] = p;
    }
    unsigned char* base = reinterpret_cast<unsigned char*>(g_noalloc_ptr[dev]);
    const bool f64 = (s->precision == 64);
    const size_t es = f64 ? 8 : 4;

    // scratch layout: work arrays of the states the solve passes through, then twiddle tables
    size_t need[2] = {0, 0};
    for (int k = 1; k < s->ndim; ++k) need[(k - 1) % 2] = std::max(need[(k - 1) % 2], s->state_reals(k, 1) * es);
    size_t off = 0;
    void* wb[2] = {nullptr, nullptr};
    for (int b = 0; b < 2; ++b) {
        if (need[b]) {
            wb[b] = base + off;
            off = align256(off + need[b]);
        }
    }

    // the passes of one solve, planned on the host with the work arrays placed in the scratch array
    void* keep[2] = {s->buf[0], s->buf[1]};
    s->buf[0] = wb[0];
    s->buf[1] = wb[1];
    s->dry = true;
    s->dry_passes.clear();
    s->dry_flags.clear();
    s->dry_names.clear();
    s->dry_fast.clear();
    s->do_fft_forward(rhs, 1);
    s->do_fft_backward_fused(field, type, 1);
    s->dry = false;
    std::vector<PassArgs> passes = s->dry_passes;
    std::vector<int> flags = s->dry_flags;
    s->dry_passes.clear();
    s->dry_flags.clear();
    s->dry_names.clear();
    s->dry_fast.clear();
    s->buf[0] = keep[0];
    s->buf[1] = keep[1];

    // twiddle tables: one per distinct (length, layout)
    std::vector<TwSlot> slots;
    auto r1_of = [&](int n) { return fast_radix1(f64 ? 1 : 0, n); };
    auto slot_for = [&](int n, int stage) -> size_t {
        for (const TwSlot& t : slots)
            if (t.n == n && t.stage == stage) return t.off;
        const int len = stage ? std::max(1, fast_stage_table_len_r1(n, stage)) : n;
        TwSlot t{n, stage, len, off};
        off = align256(off + (size_t)len * 2 * es);
        slots.push_back(t);
        return t.off;
    };
    std::vector<int> kinds(passes.size());
    for (size_t i = 0; i < passes.size(); ++i) {
        PassArgs& A = passes[i];
        const bool in64 = flags[i] & 2, out64 = flags[i] & 4;
        kinds[i] = s->fast_kind(A, f64, in64, out64);
        if (kinds[i] == 0) {
            for (int sg = 0; sg <= A.fused; ++sg) slot_for(2 * A.st[sg].M, 0);
        } else if (kinds[i] == 1) {
            slot_for(A.st[0].M, fast_radix1_mode(A.st[0].M, f64 ? 1 : 0, A.fused ? 2 : 0));
        } else if (kinds[i] == 3) {
            slot_for(A.st[0].M, fast_radix1_colreal(A.st[0].M, f64 ? 1 : 0));
        } else if (kinds[i] == 5) {
            const int M = A.st[0].M;
            slot_for(M, A.mult.mode == 2 ? fast_radix1_rowrot(M, f64 ? 1 : 0) : fast_radix1_rowfused(M, f64 ? 1 : 0));
        } else if (kinds[i] == 4) {
            const LineSpec& sp = A.st[0].spec[0];
            slot_for(2 * A.st[0].M, 0);
            if (fast_dct_family(sp.kind, sp.n_in, A.st[0].M)) {
                const int nt = fast_dct_length(sp.kind, sp.n_in, A.st[0].M);
                slot_for(nt, 0);
                slot_for(nt / 2, fast_radix1_dct(nt / 2, f64 ? 1 : 0));
            } else {
                slot_for(A.st[0].M, r1_of(A.st[0].M));
            }
        } else {
            slot_for(A.st[0].M, 0);
            slot_for(A.st[0].M / 2, fast_radix1_row(A.st[0].M / 2, f64 ? 1 : 0));
        }
    }
    if (off > FLUPS_NOALLOC_SCRATCH_BYTES) {
        char msg[256];
        snprintf(msg, sizeof(msg), "this solve needs %zu bytes of scratch, above the %u-byte limit of the no-allocation entry point",
                 off, (unsigned)FLUPS_NOALLOC_SCRATCH_BYTES);
        return fail(-3, msg);
    }

    cudaStream_t st = s->stream;
    // launch-time lookups find the slots planned above; a key that planning did
    // not place is an error (checked before anything is launched), never a new
    // slot past the size check
    bool missing = false;
    auto tw_of = [&](int n, int stage) -> const void* {
        for (const TwSlot& t : slots)
            if (t.n == n && t.stage == stage) return base + t.off;
        missing = true;
        return nullptr;
    };
    // go = false: resolve every table of every pass without launching
    auto run = [&](bool go) -> cudaError_t {
        for (size_t i = 0; i < passes.size(); ++i) {
            PassArgs A = passes[i];
            const bool in64 = flags[i] & 2, out64 = flags[i] & 4;
            cudaError_t e = cudaSuccess;
            if (kinds[i] == 0) {
                for (int sg = 0; sg <= A.fused; ++sg) A.st[sg].tw = tw_of(2 * A.st[sg].M, 0);
                if (go) e = launch_line_pass(A, f64 ? 1 : 0, in64 ? 1 : 0, out64 ? 1 : 0, st);
            } else if (kinds[i] == 5) {
                RowFusedArgs f;
                s->rowfused_args(A, f);
                const int L = A.st[0].M;
                f.tws = tw_of(L, A.mult.mode == 2 ? fast_radix1_rowrot(L, f64 ? 1 : 0) : fast_radix1_rowfused(L, f64 ? 1 : 0));
                if (go) e = launch_fast_rowfused(f64 ? 1 : 0, A.mult.mode == 2, L, f, A.ncomp, st);
            } else {
                const int L = A.st[0].M;
                ColArgs c;
                RowArgs r;
                int mode = 0;
                s->fast_args(A, kinds[i], in64, out64, c, r, mode);
                if (kinds[i] == 1) {
                    c.tws = tw_of(L, fast_radix1_mode(L, f64 ? 1 : 0, mode));
                    if (go) e = launch_fast_col(f64 ? 1 : 0, mode, L, c, A.ncomp, st);
                } else if (kinds[i] == 3) {
                    c.tws = tw_of(L, fast_radix1_colreal(L, f64 ? 1 : 0));
                    if (go) e = launch_fast_colreal(f64 ? 1 : 0, A.st[0].spec[0].kind == LK_C2R, L, c, A.ncomp, st);
                } else if (kinds[i] == 4) {
                    r.tw2 = tw_of(2 * L, 0);
                    if (fast_dct_family(r.kind, r.n, L)) {
                        const int nt = fast_dct_length(r.kind, r.n, L);
                        r.tw = tw_of(nt, 0);
                        r.tws = tw_of(nt / 2, fast_radix1_dct(nt / 2, f64 ? 1 : 0));
                    } else {
                        r.tws = tw_of(L, r1_of(L));
                    }
                    if (go) e = launch_fast_r2r(f64 ? 1 : 0, L, r, A.ncomp, st);
                } else {
                    r.tw = tw_of(L, 0);
                    r.tws = tw_of(L / 2, fast_radix1_row(L / 2, f64 ? 1 : 0));
                    if (go) e = launch_fast_row(f64 ? 1 : 0, A.st[0].spec[0].kind == LK_C2R, L, r, A.ncomp, st);
                }
            }
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    run(false);
    if (missing) return fail(-4, "a pass needs a twiddle table that was not planned (internal error)");
    for (const TwSlot& t : slots) {
        const int nb = std::min(1184, (t.len + 255) / 256);
        noalloc_twiddle_kernel<<<nb, 256, 0, st>>>(base + t.off, t.n, t.stage, t.len, t.stage, f64 ? 1 : 0);
    }
    if (const cudaError_t e = run(true); e != cudaSuccess) {
        s->last_error = (int)e;
        return fail(-4, cudaGetErrorString(e));
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        s->last_error = (int)e;
        return fail(-4, cudaGetErrorString(e));
    }
    return 0;
}
