// Solver orchestration: plans, Green's function setup, and the pass sequence
// of one solve.  Reference: src/Solver.cpp:23-202 (ctor and dry run),
// :219-469 (setup), :980-1154 (Green's function), :1207-1272 (solve),
// :1402-1542 (do_FFT / do_mult).
//
// Device data layout (every array x fastest, then y, then z, then component
// or batch):
//   state k = the field after the first k forward transforms; its extents are
//   the reference's topo_hat_[k-1] sizes, stored x fastest instead of
//   pencil-major, so no transpose is ever materialised.
//   Pass sequence for ndim directions: fwd 0 .. fwd ndim-2, one fused pass
//   (fwd ndim-1, Green multiply, bwd ndim-1) in place, bwd ndim-2 .. bwd 0.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <climits>
#include <cstring>
#include <vector>

#include "fast_dft.h"
#include "host.hpp"
#include "rot.h"

using namespace flb;

namespace flb {
int load_lgf_table(int kind, int ndim, std::vector<double>& data);
int farfield_terms(int kind, int ndim, std::vector<FarTerm>& terms, double& logc);
}  // namespace flb

static int r2r_to_line(int k) {
    switch (k) {
        case REDFT00: return LK_DCT1;
        case REDFT10: return LK_DCT2;
        case REDFT01: return LK_DCT3;
        case REDFT11: return LK_DCT4;
        case RODFT00: return LK_DST1;
        case RODFT10: return LK_DST2;
        case RODFT01: return LK_DST3;
        case RODFT11: return LK_DST4;
    }
    return LK_NONE;
}

static int fft_length(int kind, int n) {
    switch (kind) {
        case LK_DCT1: return 2 * (n - 1);
        case LK_DST1: return 2 * (n + 1);
        case LK_DCT2: case LK_DCT3: case LK_DCT4: case LK_DST2: case LK_DST3: case LK_DST4: return 2 * n;
        default: return n;
    }
}

static void factorize(int M, LineStage& S) {
    S.nrad = 0;
    int m = M;
    const int pref[4] = {16, 8, 4, 2};
    for (int r : pref) {
        while (m % r == 0 && m > 1) {
            FLB_CHECK(S.nrad < kMaxRadices, "too many FFT stages");
            S.radix[S.nrad++] = r;
            m /= r;
        }
    }
    for (int p = 3; m > 1; p += 2) {
        while (m % p == 0) {
            FLB_CHECK(p <= 64, "transform length %d has a prime factor %d > 64 (not supported)", M, p);
            FLB_CHECK(S.nrad < kMaxRadices, "too many FFT stages");
            S.radix[S.nrad++] = p;
            m /= p;
        }
    }
    if (S.nrad == 0) S.radix[S.nrad++] = 1;
}

// ---------------------------------------------------------------------------
Solver::Solver(Topology* t, FLUPS_BoundaryType* bcin[3][2], const double hin[3], const double Lin[3], int od, const int ctr[3],
               Profiler* p)
    : topo_phys(t), odiff(od), prof(p) {
    FLB_CHECK(t != nullptr, "topology is NULL");
    FLB_CHECK(t->nproc[0] * t->nproc[1] * t->nproc[2] == 1, "this library runs on a size-1 communicator");
    FLB_CHECK(!t->nf || t->nf == 1, "The RHS topology cannot be complex");
    FLB_CHECK(ctr[0] == ctr[1] && ctr[0] == ctr[2], "We handle only data located at the same place in all the direction");
    lda = t->lda;
    FLB_CHECK(lda >= 1 && lda <= 3, "lda must be 1, 2 or 3");
    center = ctr[0];
    for (int d = 0; d < 3; ++d) {
        h[d] = hin[d];
        L[d] = Lin[d];
        for (int s = 0; s < 2; ++s)
            for (int c = 0; c < lda; ++c) bc[d][s][c] = bcin[d][s][c];
    }
    for (int d = 0; d < 3; ++d) {
        fwd[d] = DirPlan(lda, d, h, L, bc[d][0], bc[d][1], FLUPS_FORWARD, false, center);
        bwd[d] = DirPlan(lda, d, h, L, bc[d][0], bc[d][1], FLUPS_BACKWARD, false, center);
        grn[d] = DirPlan(1, d, h, L, bc[d][0], bc[d][1], FLUPS_FORWARD, true, center);
    }
    sort_plans(fwd);
    sort_plans(bwd);
    sort_plans(grn);
    if (odiff != NOD) {
        // Solver.cpp:86-143: backward plans of the derivative swap EVEN and ODD
        have_diff = true;
        for (int id = 0; id < 3; ++id) {
            const int d = bwd[id].dim;
            int l[3], r[3];
            for (int c = 0; c < lda; ++c) {
                auto sw = [](int b) { return b == EVEN ? ODD : (b == ODD ? EVEN : b); };
                l[c] = sw(bc[d][0][c]);
                r[c] = sw(bc[d][1][c]);
            }
            dif[id] = DirPlan(lda, d, h, L, l, r, FLUPS_BACKWARD, false, center);
        }
    }
    ndim = 0;
    for (int d = 0; d < 3; ++d)
        if (fwd[d].type != EMPTY) ++ndim;
    FLB_CHECK(ndim > 1, "We only hanlde 2D and 3D field");
    dry_run(fwd);
    {
        // states of the field after each forward transform
        st[0].cplx = false;
        for (int d = 0; d < 3; ++d) st[0].n[d] = t->nglob[d];
        for (int ip = 0; ip < ndim; ++ip) {
            st[ip + 1] = st[ip];
            st[ip + 1].n[fwd[ip].dim] = fwd[ip].n_out;
            st[ip + 1].cplx = st[ip].cplx || fwd[ip].isr2c;
        }
    }
    dry_run(bwd);
    dry_run(grn);
    if (have_diff) dry_run(dif);
    normfact = 1.0;
    volfact = 1.0;
    for (int ip = 0; ip < 3; ++ip) {
        normfact *= fwd[ip].normfact;
        volfact *= fwd[ip].volfact;
    }
    build_xlast();
}

// The x-last plans of an all-unbounded 3-D problem (see host.hpp): the same
// per-direction tables (FFTW_plan_dim_{cell,node}.cpp) initialised in the
// order z, y, x, so z becomes the real-to-complex direction.
void Solver::build_xlast() {
    if (ndim != 3) return;
    // every direction unbounded or periodic: z, y, x is then a valid order of
    // the same transforms (the Green's spectrum is even in each direction and
    // folds to the same extents in both orders; compute_green checks it)
    xlast_mixed = false;
    for (int ip = 0; ip < 3; ++ip) {
        if (fwd[ip].type == PERPER) xlast_mixed = true;
        else if (fwd[ip].type != UNBUNB) return;
    }
    const int order[3] = {2, 1, 0};
    for (int k = 0; k < 3; ++k) {
        const int d = order[k];
        xfwd[k] = DirPlan(lda, d, h, L, bc[d][0], bc[d][1], FLUPS_FORWARD, false, center);
        xbwd[k] = DirPlan(lda, d, h, L, bc[d][0], bc[d][1], FLUPS_BACKWARD, false, center);
        if (have_diff) {
            int l[3], r[3];
            for (int c = 0; c < lda; ++c) {
                auto sw = [](int b) { return b == EVEN ? ODD : (b == ODD ? EVEN : b); };
                l[c] = sw(bc[d][0][c]);
                r[c] = sw(bc[d][1][c]);
            }
            xdif[k] = DirPlan(lda, d, h, L, l, r, FLUPS_BACKWARD, false, center);
        }
    }
    dry_run(xfwd);
    dry_run(xbwd);
    if (have_diff) dry_run(xdif);
    xst[0] = st[0];
    for (int ip = 0; ip < ndim; ++ip) {
        xst[ip + 1] = xst[ip];
        xst[ip + 1].n[xfwd[ip].dim] = xfwd[ip].n_out;
        xst[ip + 1].cplx = xst[ip].cplx || xfwd[ip].isr2c;
    }
    has_xlast = true;
}

void Solver::swap_order() {
    for (int k = 0; k < 3; ++k) {
        std::swap(fwd[k], xfwd[k]);
        std::swap(bwd[k], xbwd[k]);
        std::swap(dif[k], xdif[k]);
        std::swap(gfold_M[k], xgfold_M[k]);
    }
    for (int k = 0; k < 4; ++k) std::swap(st[k], xst[k]);
    std::swap(ksym, xksym);
    std::swap(kstr, xkstr);
    xlast_active = !xlast_active;
}

// The x-last order runs when every pass of it has a register-DFT kernel and
// the fused pass is the row kernel (planned on the host at set-up, per
// solver type).
bool Solver::xlast_ok(int type) const {
    if (!has_xlast || !xlast_on || !use_fast || owned() || slab_dim >= 0 || xlast_active) return false;
    return xlast_fast[type == ROT ? 1 : 0];
}

void Solver::plan_xlast() {
    xlast_fast[0] = xlast_fast[1] = false;
    if (!has_xlast) return;
    for (int t = 0; t < 2; ++t) {
        const int type = t ? ROT : STD;
        // ROT: the fused rows' Nyquist treatment reproduces the spectrum of a
        // reference order whose real-to-complex direction is x; with a
        // periodic direction that holds when x is the reference's first
        // direction (periodic x), else the reference's order stays
        if (type == ROT && (lda != 3 || !have_diff || (xlast_mixed && fwd[0].dim != 0))) continue;
        swap_order();
        const bool keep = dry;
        dry = true;
        dry_passes.clear();
        dry_flags.clear();
        dry_names.clear();
        dry_fast.clear();
        do_fft_forward(nullptr, 1);
        do_fft_backward_fused(nullptr, type, 1);
        bool ok = !dry_fast.empty();
        for (size_t i = 0; i < dry_fast.size(); ++i) {
            if (dry_fast[i] == 0) ok = false;
            if (dry_passes[i].fused && dry_fast[i] != 5) ok = false;
        }
        dry_passes.clear();
        dry_flags.clear();
        dry_names.clear();
        dry_fast.clear();
        dry = keep;
        swap_order();
        xlast_fast[t] = ok;
    }
}

void Solver::dry_run(DirPlan p[3]) {
    // Solver.cpp:617-650
    int size[3] = {topo_phys->nglob[0], topo_phys->nglob[1], topo_phys->nglob[2]};
    bool cplx = false;
    for (int ip = 0; ip < ndim; ++ip) {
        if (&p[0] == &fwd[0])
            for (int d = 0; d < 3; ++d) sizes_before[ip][d] = size[d];
        p[ip].init(size, cplx);
        size[p[ip].dim] = p[ip].n_out;
        cplx = cplx || p[ip].isr2c;
    }
}

Solver::~Solver() {
    group_forget(this);
    drop_graphs();
    if (ov_stream[0]) {
        for (int i = 0; i < 2; ++i) {
            cudaStreamSynchronize(ov_stream[i]);
            cudaStreamDestroy(ov_stream[i]);
        }
        cudaEventDestroy(ov_ev0);
        for (int k = 0; k < kOvSlabs; ++k) {
            cudaEventDestroy(ov_evf[k]);
            cudaEventDestroy(ov_evg[k]);
        }
    }
    if (capture_stream) cudaStreamDestroy(capture_stream);
    if (h2d_stream) {
        // copies and passes of an async solve may still be in flight
        cudaStreamSynchronize(h2d_stream);
        cudaStreamSynchronize(d2h_stream);
        if (cstream) cudaStreamSynchronize(cstream);
    }
    for (auto& b : buf)
        if (b) cudaFree(b);
    if (xbuf) cudaFree(xbuf);
    if (green_share) cudaFree(green_share);
    else if (green) cudaFree(green);
    for (auto& kv : twiddles) cudaFree(kv.second);
    if (stage_in) cudaFree(stage_in);
    if (stage_out) cudaFree(stage_out);
    if (xlast_active) swap_order();
    if (ksym) cudaFree(ksym);
    if (xksym) cudaFree(xksym);
    if (h2d_stream) {
        for (int k = 0; k < kSlabs; ++k) {
            cudaEventDestroy(ev_in[k]);
            cudaEventDestroy(ev_fwd[k]);
            cudaEventDestroy(ev_bwd[k]);
            cudaEventDestroy(ev_out[k]);
        }
        cudaStreamDestroy(h2d_stream);
        cudaStreamDestroy(d2h_stream);
        if (cstream) cudaStreamDestroy(cstream);
        if (ev_entry) cudaEventDestroy(ev_entry);
    }
    if (inner) cudaFree(inner);
    for (auto e : ev) cudaEventDestroy(e);
    delete topo_spec;
    delete topo_inner_phys;
}

void Solver::check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        last_error = (int)e;
        FLB_CHECK(false, "CUDA error during %s: %s", what, cudaGetErrorString(e));
    }
}

void Solver::spectral_info(double kf[3], double ko[3], double ss[3]) const {
    // Solver.hpp:222-229
    for (int ip = 0; ip < 3; ++ip) {
        const int d = fwd[ip].dim;
        kf[d] = fwd[ip].kfact;
        ss[d] = fwd[ip].symstart;
        ko[d] = fwd[ip].koffset;
    }
}

size_t Solver::alloc_size() const {
    size_t m = 1;
    for (int k = 1; k <= ndim; ++k) {
        size_t e = (size_t)st[k].n[0] * st[k].n[1] * st[k].n[2] * (st[k].cplx ? 2 : 1) * lda;
        m = std::max(m, e);
    }
    return std::max(m, topo_phys->memsize());
}

const void* Solver::twiddle(int M, bool f64) {
    const int64_t key = (int64_t)M * 2 + (f64 ? 1 : 0);
    auto it = twiddles.find(key);
    if (it != twiddles.end()) return it->second;
    // W_{2M}^q = exp(-2 pi i q / (2M)), q in [0, 2M), evaluated in FP64
    std::vector<double> w(4 * (size_t)M);
    for (int q = 0; q < 2 * M; ++q) {
        // reduce to the first quadrant for accuracy: angle = -pi q / M
        const long double a = -(long double)M_PI * (long double)q / (long double)M;
        w[2 * q] = (double)cosl(a);
        w[2 * q + 1] = (double)sinl(a);
    }
    void* d = nullptr;
    if (f64) {
        check_cuda(cudaMalloc(&d, w.size() * sizeof(double)), "twiddle allocation");
        check_cuda(cudaMemcpy(d, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice), "twiddle upload");
    } else {
        std::vector<float> wf(w.size());
        for (size_t i = 0; i < w.size(); ++i) wf[i] = (float)w[i];
        check_cuda(cudaMalloc(&d, wf.size() * sizeof(float)), "twiddle allocation");
        check_cuda(cudaMemcpy(d, wf.data(), wf.size() * sizeof(float), cudaMemcpyHostToDevice), "twiddle upload");
    }
    twiddles[key] = d;
    return d;
}

// ---------------------------------------------------------------- stages
LineStage Solver::stage_forward(const DirPlan& p, int ip, bool f64) {
    LineStage S;
    memset(&S, 0, sizeof(S));
    int M = -1;
    for (int c = 0; c < p.lda; ++c) {
        LineSpec& sp = S.spec[c];
        if (p.type == SYMSYM || p.type == MIXUNB) {
            sp.kind = r2r_to_line(p.kind[c]);
            sp.n_in = p.n_in[c];
        } else {
            sp.kind = p.isr2c ? LK_R2C : LK_C2C;
            sp.n_in = p.n_in[0];
        }
        sp.sign = -1;
        sp.fi = p.fstart_in[c];
        sp.fo = p.fstart_out[c];
        sp.postpro = p.postpro[c];
        sp.nfftw = p.n_out - 1;
        const int m = fft_length(sp.kind, sp.n_in);
        FLB_CHECK(M < 0 || M == m, "components need transforms of the same length");
        M = m;
    }
    for (int c = p.lda; c < kMaxComp; ++c) S.spec[c] = S.spec[0];
    S.M = M;
    factorize(M, S);
    S.n_b = p.isr2c ? 2 * p.n_out : p.n_out;
    S.fieldstart = p.fieldstart;
    S.n_o = p.n_out;
    S.in_cplx = (ip >= 0) ? st[ip].cplx : 0;
    S.out_cplx = (ip >= 0) ? st[ip + 1].cplx : 0;
    S.store_off = 0;
    S.n_store = S.n_o;
    S.tw = nullptr;  // resolved at launch
    return S;
}

LineStage Solver::stage_backward(const DirPlan& p, const DirPlan& pf, int ip, bool f64) {
    LineStage S;
    memset(&S, 0, sizeof(S));
    int M = -1;
    for (int c = 0; c < p.lda; ++c) {
        LineSpec& sp = S.spec[c];
        if (p.type == SYMSYM || p.type == MIXUNB) {
            sp.kind = r2r_to_line(p.kind[c]);
            sp.n_in = p.n_in[c];
        } else {
            sp.kind = pf.isr2c ? LK_C2R : LK_C2C;
            sp.n_in = p.n_in[0];
        }
        sp.sign = +1;
        sp.fi = p.fstart_in[c];
        sp.fo = p.fstart_out[c];
        sp.postpro = p.postpro[c];
        sp.nfftw = p.n_in[c];
        const int m = fft_length(sp.kind, sp.n_in);
        FLB_CHECK(M < 0 || M == m, "components need transforms of the same length");
        M = m;
    }
    for (int c = p.lda; c < kMaxComp; ++c) S.spec[c] = S.spec[0];
    S.M = M;
    factorize(M, S);
    S.n_b = p.n_out;
    S.fieldstart = 0;
    S.n_o = pf.isr2c ? 2 * p.n_out : p.n_out;
    S.in_cplx = st[ip + 1].cplx;
    S.out_cplx = st[ip].cplx;
    S.store_off = pf.fieldstart;
    S.n_store = st[ip].n[pf.dim];
    S.tw = nullptr;  // resolved at launch
    return S;
}

// Work arrays keep every x row on a 128-byte boundary (the x extent, e.g. N+1
// complex after an r2c, is padded in memory; the padding is never read or
// written), so that the 32-byte sectors of a warp's row segment are whole.
int64_t Solver::row_pitch(const ArrState& s) const {
    const int64_t eb = (int64_t)(precision == 64 ? 8 : 4) * (s.cplx ? 2 : 1);
    const int64_t q = std::max<int64_t>(1, 128 / eb);
    return ((int64_t)s.n[0] + q - 1) / q * q;
}

size_t Solver::state_reals(int k, int nbatch) const {
    return (size_t)row_pitch(st[k]) * st[k].n[1] * st[k].n[2] * (st[k].cplx ? 2 : 1) * lda * nbatch;
}

// reals of work array b (0: states 1, 3, ...; 1: states 2, ...) for nbatch
// right-hand sides: the larger of the two pass orders when both exist
size_t Solver::work_reals(int b, int nbatch) const {
    size_t need = 0;
    for (int k = 1; k < ndim; ++k) {
        if ((k - 1) % 2 != b) continue;
        size_t r = state_reals(k, nbatch);
        if (owned()) r = r / (size_t)st[k].n[2] * (size_t)(own[1] - own[0]);
        need = std::max(need, r);
        if (has_xlast && !owned()) {
            const ArrState& X = xst[k];
            need = std::max(need, (size_t)row_pitch(X) * X.n[1] * X.n[2] * (X.cplx ? 2 : 1) * lda * nbatch);
        }
    }
    return need;
}

void Solver::set_strides_internal(int64_t str[3], int64_t& cstr, const ArrState& s, bool pad) const {
    const int64_t px = pad ? row_pitch(s) : s.n[0];
    str[0] = 1;
    str[1] = px;
    str[2] = px * s.n[1];
    cstr = px * s.n[1] * s.n[2];
}

void Solver::set_strides_user(int64_t str[3], int64_t& cstr) const {
    // flups_locID layout of the user topology (src/flups.h:109-119)
    const Topology* t = topo_phys;
    const int a0 = t->axis, a1 = (a0 + 1) % 3, a2 = (a0 + 2) % 3;
    str[a0] = 1;
    str[a1] = t->nmem[a0];
    str[a2] = (int64_t)t->nmem[a0] * t->nmem[a1];
    cstr = (int64_t)t->memdim();
}

PassArgs Solver::base_pass(int axis, const ArrState& src, int ncomp, int lda_spec) {
    PassArgs A;
    memset(&A, 0, sizeof(A));
    A.axis = axis;
    A.n_src = src.n[axis];
    const int a = (axis == 0) ? 1 : 0, b = (axis == 2) ? 1 : 2;
    A.n_a = src.n[a];
    A.n_b = src.n[b];
    A.nlines = A.n_a * A.n_b;
    A.ncomp = ncomp;
    A.lda = lda_spec;
    return A;
}

void Solver::fit_lines(PassArgs& A, int elem_bytes) const {
    A.lines_per_cta = 1;
    const size_t one = line_pass_smem(A, elem_bytes);
    FLB_CHECK(one <= 227 * 1024, "a line of this size does not fit in shared memory (%zu bytes)", one);
    // tiles of about 50 KB (FP32, 4 CTAs per SM) or 100 KB (FP64, whose
    // register count allows 2): several resident CTAs hide the barriers of
    // the shared-memory stages
    const size_t target = (elem_bytes == 4 ? 50 : 100) * 1024;
    int tl = (int)std::min<size_t>(32, target / one);
    tl = std::max(tl, 1);
    const int64_t work = A.comps_together ? A.nlines : (int64_t)A.nlines * A.ncomp;
    if (tl > work) tl = (int)std::max<int64_t>(1, work);
    A.lines_per_cta = tl;
}

MultSpec Solver::mult_spec(int type) const {
    MultSpec G;
    memset(&G, 0, sizeof(G));
    G.mode = (type == ROT) ? 2 : 1;
    G.green = green;
    for (int d = 0; d < 3; ++d) {
        G.gstr[d] = gstr[d];
        G.gfold[d] = gfold_M[d];
        G.gn[d] = gfold_n[d];
        G.hgrid[d] = h[d];
    }
    G.normfact = 1.0;  // already in the stored spectrum (compute_green)
    G.odiff = odiff;
    if (type == ROT) {
        double kabs[3], ko[3], ss[3];
        spectral_info(kabs, ko, ss);
        for (int d = 0; d < 3; ++d) {
            G.koffset[d] = ko[d];
            G.symstart[d] = ss[d];
        }
        // Solver.cpp:1485-1516: phase of the derivative from the forward and backward-diff imult
        for (int ip = 0; ip < 3; ++ip) {
            const int d = fwd[ip].dim;
            for (int c = 0; c < 3; ++c) {
                const int cc = c < lda ? c : 0;
                int ph = 0;
                if (fwd[ip].imult[cc]) ph--;
                if (dif[ip].imult[cc]) ph++;
                if (ph == 0) { G.kfact[d][c][0] = 0.0; G.kfact[d][c][1] = kabs[d]; }
                else if (ph == 1) { G.kfact[d][c][0] = -kabs[d]; G.kfact[d][c][1] = 0.0; }
                else { G.kfact[d][c][0] = kabs[d]; G.kfact[d][c][1] = 0.0; }
            }
        }
    }
    return G;
}

// Which register-resident kernel can run this pass (0 = none: the general line pass).
int Solver::fast_kind(const PassArgs& A, bool f64, bool in_f64, bool out_f64) const {
    if (!use_fast) return 0;
    // components together: only the fused ROT pass (groups of three components)
    const bool rot = A.fused && A.mult.mode == 2;
    // (the curl tables exist once set up; host-only planning assumes them)
    if (A.comps_together && !(rot && A.lda == 3 && A.ncomp % 3 == 0 && (ksym || dry))) return 0;
    if (rot && !A.comps_together) return 0;
    if (A.n_b > 65535 || A.ncomp > 65535) return 0;  // grid y / z limits of the fast launches
    // vector loads/stores of complex (or real pairs) need their natural alignment
    const uintptr_t ain = dry ? 0 : (uintptr_t)A.in, aout = dry ? 0 : (uintptr_t)A.out;
    if ((ain % (in_f64 ? 16 : 8)) != 0 || (aout % (out_f64 ? 16 : 8)) != 0) return 0;
    {
        const LineStage& S0 = A.st[0];
        const int k0 = S0.spec[0].kind;
        if (A.axis != 0 && !A.fused && (k0 == LK_R2C || k0 == LK_C2R)) {
            // columns of a real transform (r2c forward, c2r backward), working precision;
            // the node-centred periodic copy (PP_ENFORCE_PERIOD of index nfftw from 0) in the kernel
            const int L = S0.M;
            const LineSpec& sp0 = S0.spec[0];
            for (int c = 0; c < A.lda; ++c) {
                const LineSpec& sp = S0.spec[c];
                // (nfftw only matters to the periodic copy)
                if (sp.kind != k0 || sp.n_in != sp0.n_in || sp.fi != 0 || sp.fo != 0 || sp.postpro != sp0.postpro ||
                    (sp0.postpro == PP_ENFORCE_PERIOD && sp.nfftw != sp0.nfftw))
                    return 0;
            }
            if (sp0.postpro != PP_NONE && sp0.postpro != PP_ENFORCE_PERIOD) return 0;
            const int extra = (sp0.postpro == PP_ENFORCE_PERIOD) ? 1 : 0;
            if (S0.fieldstart != 0 || S0.store_off != 0) return 0;
            if (!fast_col_supported(L)) return 0;
            // the complex side is in the working precision; the real side is too, or
            // it is the user's doubles (first or last pass of an FP32 solve)
            if ((k0 == LK_R2C ? out_f64 : in_f64) != f64) return 0;
            if (f64 && (k0 == LK_R2C ? !in_f64 : !out_f64)) return 0;
            if (A.in_str[0] != 1 || A.out_str[0] != 1) return 0;
            if ((int64_t)(L + 1) * A.in_str[A.axis] >= (int64_t)INT32_MAX || (int64_t)(L + 1) * A.out_str[A.axis] >= (int64_t)INT32_MAX)
                return 0;
            if (k0 == LK_R2C) {
                if (S0.in_cplx || !S0.out_cplx || A.n_src > L + extra || S0.n_store != L / 2 + 1 + extra) return 0;
                if (extra && sp0.nfftw != L / 2 + 1) return 0;
            } else {
                if (!S0.in_cplx || S0.out_cplx || A.n_src != L / 2 + 1 + extra || S0.n_store > L + extra) return 0;
                if (extra && (sp0.nfftw != L || S0.n_store != L + 1)) return 0;
            }
            return 3;
        }
        // r2r rows (DCT / DST I-IV): the post-processing is done by the kernel
        if (k0 >= LK_DCT1 && k0 <= LK_DST4) {
            if (A.fused || A.axis != 0) return 0;
            const bool half = fast_dct_family(k0, S0.spec[0].n_in, S0.M) != 0;
            if (!fast_r2r_supported(S0.M) && !half) return 0;
            // the half-length kernels place the transform at fi / fo in its row
            // (node-centred DST-I: the boundary values stay outside); the
            // M-point kernel does not
            if (!half && (S0.spec[0].fi != 0 || S0.spec[0].fo != 0)) return 0;
            for (int c = 0; c < A.lda; ++c) {
                const LineSpec& sp = S0.spec[c];
                if (sp.kind != k0 || sp.n_in != S0.spec[0].n_in || sp.fi != S0.spec[0].fi || sp.fo != S0.spec[0].fo ||
                    sp.postpro != S0.spec[0].postpro || sp.nfftw != S0.spec[0].nfftw)
                    return 0;
            }
            if (S0.fieldstart != 0 || S0.store_off != 0 || S0.in_cplx || S0.out_cplx) return 0;
            if (A.n_src > S0.M || S0.n_store > S0.M || A.in_str[0] != 1 || A.out_str[0] != 1) return 0;
            if (f64 && (!in_f64 || !out_f64)) return 0;
            return 4;
        }
    }
    const int nst = A.fused ? 2 : 1;
    for (int s2 = 0; s2 < nst; ++s2) {
        const LineStage& S = A.st[s2];
        for (int c = 0; c < A.lda; ++c) {
            const LineSpec& sp = S.spec[c];
            if (sp.fi != 0 || sp.fo != 0 || sp.postpro != PP_NONE) return 0;
            if (sp.kind != S.spec[0].kind || sp.n_in != S.spec[0].n_in) return 0;
        }
        if (S.fieldstart != 0 || S.store_off != 0) return 0;
    }
    const LineStage& S0 = A.st[0];
    const int k0 = S0.spec[0].kind;
    if (A.axis != 0) {
        // columns: complex DFT, working precision in and out, x contiguous
        if (k0 != LK_C2C || !S0.in_cplx || !S0.out_cplx || in_f64 != f64 || out_f64 != f64) return 0;
        if (A.fused && (A.st[1].spec[0].kind != LK_C2C || A.st[1].M != S0.M || (A.mult.mode != 1 && !rot))) return 0;
        if (A.fused && (A.mult.gfold[A.axis] != S0.M || (int64_t)S0.M * A.mult.gstr[A.axis] >= (int64_t)INT32_MAX)) return 0;
        if (A.in_str[0] != 1 || A.out_str[0] != 1) return 0;
        const int L = S0.M;
        if (!fast_col_supported(L) || A.n_src > L) return 0;
        // 32-bit element offsets along a line
        if ((int64_t)L * A.in_str[A.axis] >= (int64_t)INT32_MAX || (int64_t)L * A.out_str[A.axis] >= (int64_t)INT32_MAX) return 0;
        const LineStage& SL = A.st[A.fused ? 1 : 0];
        if (SL.n_store > L) return 0;
        if (!A.fused && S0.n_o != L) return 0;
        return 1;
    }
    if (A.fused) {
        // the last direction along x: the fused row pass (one warp per row)
        if (k0 != LK_C2C || !S0.in_cplx || !S0.out_cplx || in_f64 != f64 || out_f64 != f64) return 0;
        const int L = S0.M;
        if (A.st[1].spec[0].kind != LK_C2C || A.st[1].M != L || (A.mult.mode != 1 && !rot)) return 0;
        if (!fast_rowfused_supported(f64 ? 1 : 0, L) || A.n_src > L || A.st[1].n_store > L) return 0;
        if (A.in_str[0] != 1 || A.out_str[0] != 1 || A.in != A.out) return 0;
        for (int d = 0; d < 3; ++d)
            if (A.in_str[d] != A.out_str[d]) return 0;
        if (A.mult.gfold[0] != L || A.mult.gstr[0] != 1 || A.mult.gstr[1] < L / 2 + 4) return 0;
        const int64_t es = f64 ? 8 : 4;
        if ((A.mult.gstr[1] * es) % 16 != 0 || (A.mult.gstr[2] * es) % 16 != 0) return 0;
        if (!dry && (reinterpret_cast<uintptr_t>(A.mult.green) & 15) != 0) return 0;
        return 5;
    }
    const int L = S0.M;
    if (!fast_row_supported(L) || A.in_str[0] != 1 || A.out_str[0] != 1) return 0;
    auto even = [](int64_t v) { return (v % 2) == 0; };
    if (k0 == LK_R2C) {
        if (S0.in_cplx || !S0.out_cplx || A.n_src > L || S0.n_o != L / 2 + 1 || S0.n_store != S0.n_o) return 0;
        if (!even(A.in_str[1]) || !even(A.in_str[2]) || !even(A.in_cstr)) return 0;
        if (out_f64 != f64) return 0;
        return 2;
    }
    if (k0 == LK_C2R) {
        if (!S0.in_cplx || S0.out_cplx || A.n_src != L / 2 + 1 || S0.n_store > L) return 0;
        if (!even(A.out_str[1]) || !even(A.out_str[2]) || !even(A.out_cstr)) return 0;
        if (in_f64 != f64) return 0;
        return 2;
    }
    return 0;
}

void Solver::fast_args(const PassArgs& A, int kind, bool in_f64, bool out_f64, ColArgs& c, RowArgs& r, int& mode) const {
    const LineStage& S0 = A.st[0];
    const int b = (A.axis == 2) ? 1 : 2;
    memset(&c, 0, sizeof(c));
    memset(&r, 0, sizeof(r));
    mode = 0;
    if (kind == 1 || kind == 3) {
        c.in = A.in;
        c.out = A.out;
        c.nx = A.n_a;
        c.nouter = A.n_b;
        c.nin = A.n_src;
        c.nout = A.st[A.fused ? 1 : 0].n_store;
        c.period = (kind == 3 && A.st[0].spec[0].postpro == PP_ENFORCE_PERIOD) ? A.st[0].spec[0].nfftw : -1;
        if (kind == 3) {
            c.real64 = (S0.spec[0].kind == LK_R2C) ? (in_f64 && !out_f64) : (out_f64 && !in_f64);
            // neighbouring columns two at a time when every pair is aligned
            auto even = [](int64_t v) { return (v % 2) == 0; };
            const bool strides = even(A.in_str[1]) && even(A.in_str[2]) && even(A.in_cstr) && even(A.out_str[1]) &&
                                 even(A.out_str[2]) && even(A.out_cstr);
            const bool bases = dry || ((reinterpret_cast<uintptr_t>(A.in) & 15) == 0 && (reinterpret_cast<uintptr_t>(A.out) & 15) == 0);
            c.pairs = (strides && bases) ? 1 : 0;
        }
        c.in_lstr = A.in_str[A.axis];
        c.in_ostr = A.in_str[b];
        c.in_cstr = A.in_cstr;
        c.out_lstr = A.out_str[A.axis];
        c.out_ostr = A.out_str[b];
        c.out_cstr = A.out_cstr;
        mode = (S0.spec[0].sign > 0) ? 1 : 0;
        if (A.fused) {
            mode = (A.mult.mode == 2) ? 3 : 2;
            if (mode == 3) {
                c.ksym = ksym;
                c.kstr = kstr;
                c.ax_line = A.axis;
                c.ax_outer = b;
            }
            c.green = A.mult.green;
            c.g_x = A.mult.gstr[0];
            c.g_line = A.mult.gstr[A.axis];
            c.g_outer = A.mult.gstr[b];
            c.f_x = A.mult.gfold[0];
            c.f_line = A.mult.gfold[A.axis];
            c.f_outer = A.mult.gfold[b];
            c.normfact = A.mult.normfact;
        }
        return;
    }
    r.in = A.in;
    r.out = A.out;
    r.n1 = A.n_a;
    r.nrows = A.n_a * A.n_b;
    r.nin = A.n_src;
    r.nout = S0.n_store;
    r.kind = S0.spec[0].kind;
    r.n = S0.spec[0].n_in;
    r.nstore = S0.n_store;
    r.postpro = S0.spec[0].postpro;
    r.nfftw = S0.spec[0].nfftw;
    r.fi = S0.spec[0].fi;
    r.fo = S0.spec[0].fo;
    r.ilast = S0.n_o - 1;
    r.in_s1 = A.in_str[1];
    r.in_s2 = A.in_str[2];
    r.in_cstr = A.in_cstr;
    r.out_s1 = A.out_str[1];
    r.out_s2 = A.out_str[2];
    r.out_cstr = A.out_cstr;
    r.in_f64 = in_f64;
    r.out_f64 = out_f64;
}

// arguments of the fused row pass (kind 5): rows (y, z) of the x-fastest array
void Solver::rowfused_args(const PassArgs& A, RowFusedArgs& f) const {
    memset(&f, 0, sizeof(f));
    f.in = A.in;
    f.out = A.out;
    f.n1 = A.n_a;
    f.n2 = A.n_b;
    f.nin = A.n_src;
    f.nout = A.st[1].n_store;
    f.s1 = A.in_str[1];
    f.s2 = A.in_str[2];
    f.cstr = A.in_cstr;
    f.green = A.mult.green;
    f.g1 = A.mult.gstr[1];
    f.g2 = A.mult.gstr[2];
    f.f1 = A.mult.gfold[1];
    f.f2 = A.mult.gfold[2];
    if (A.mult.mode == 2) {
        f.ksym = ksym;
        f.kstr = kstr;
        f.ax1 = 1;
        f.ax2 = 2;
        // the Nyquist index of each direction: half its DFT length
        for (int ip = 0; ip < ndim; ++ip) {
            const DirPlan& p = fwd[ip];
            f.nyq[p.dim] = (p.type == PERPER || p.type == UNBUNB) ? (p.isr2c ? p.n_out - 1 : p.n_in[0] / 2) : -1;
        }
        for (int d = ndim; d < 3; ++d) f.nyq[fwd[d].dim] = -1;
    }
}

void Solver::launch_fast(const PassArgs& A, int kind, bool f64, bool in_f64, bool out_f64) {
    const int L = A.st[0].M;
    if (kind == 5) {
        RowFusedArgs f;
        rowfused_args(A, f);
        f.tws = stage_table(L, f64, A.mult.mode == 2 ? fast_radix1_rowrot(L, f64 ? 1 : 0) : fast_radix1_rowfused(L, f64 ? 1 : 0));
        if (prefetch && A.mult.mode == 2) rowrot_prefetch(f, f64, L, A.ncomp);
        check_cuda(launch_fast_rowfused(f64 ? 1 : 0, A.mult.mode == 2, L, f, A.ncomp, stream), "fused row launch");
        return;
    }
    ColArgs c;
    RowArgs r;
    int mode = 0;
    fast_args(A, kind, in_f64, out_f64, c, r, mode);
    if (kind == 4) {
        r.tw2 = twiddle(L, f64);
        if (fast_dct_family(r.kind, r.n, L)) {
            const int nt = fast_dct_length(r.kind, r.n, L);
            r.tw = twiddle_plain(nt, f64);
            r.tws = stage_table(nt / 2, f64, fast_radix1_dct(nt / 2, f64 ? 1 : 0));
        } else {
            r.tws = stage_table(L, f64);
        }
        check_cuda(launch_fast_r2r(f64, L, r, A.ncomp, stream), "r2r row launch");
        return;
    }
    if (kind == 3) {
        c.tws = stage_table(L, f64, fast_radix1_colreal(L, f64 ? 1 : 0));
        check_cuda(launch_fast_colreal(f64, A.st[0].spec[0].kind == LK_C2R, L, c, A.ncomp, stream), "column r2c/c2r launch");
        return;
    }
    if (kind == 1) {
        c.tws = stage_table(L, f64, fast_radix1_mode(L, f64 ? 1 : 0, mode));
        if (force_tile) {
            c.tile = force_tile;
        } else if (!tuned_tile.empty()) {
            auto it = tuned_tile.find(pass_key(A, f64));
            if (it != tuned_tile.end()) c.tile = it->second;
        }
        if (prefetch && mode < 2) col_prefetch(c, f64, L, A.ncomp);
        if (peers.n > 0 && owned() && slab_dim == 2 && A.axis == 1 && mode < 2 && A.ncomp == 1) {
            // a share's y pass: outputs (forward) or inputs (inverse) in the owners' column arrays
            c.peers = peers;
            c.peers.zs = own[0];
            c.peers.nl = st[ndim - 1].n[1];
            if (mode == 1) c.pf.nbox = 0;
        }
        check_cuda(launch_fast_col(f64, mode, L, c, A.ncomp, stream), "column DFT launch");
        return;
    }
    r.tw = twiddle_plain(L, f64);
    r.tws = stage_table(L / 2, f64, fast_radix1_row(L / 2, f64 ? 1 : 0));
    const bool c2r = A.st[0].spec[0].kind == LK_C2R;
    if (prefetch) row_prefetch(r, f64, c2r, L, A.ncomp);
    check_cuda(launch_fast_row(f64, c2r, L, r, A.ncomp, stream), "row DFT launch");
}

// L2 prefetch of the next blocks' input for the forward / inverse column
// passes along a short-stride axis (lines farther apart than 64 KB touch a
// DRAM page per element and gain nothing) and for the r2c / c2r rows.
static constexpr int PREFETCH_DIST = 148;
// inputs smaller than this stay in the 126 MB L2 anyway: no tensor map is built
static constexpr double PREFETCH_MIN_BYTES = 64.0 * 1024 * 1024;

void Solver::col_prefetch(ColArgs& c, bool f64, int L, int ncomp) const {
    const int es = f64 ? 16 : 8, u = es / 8;
    if ((int64_t)c.in_lstr * es > 65536) return;
    if ((double)c.nx * c.nin * c.nouter * ncomp * es < PREFETCH_MIN_BYTES) return;
    const int tx = fast_col_tile_width(f64 ? 1 : 0, L, c.tile);
    const uint64_t outer_bytes = (uint64_t)c.in_ostr * es;
    const uint64_t dims[4] = {(uint64_t)c.nx * u, (uint64_t)c.nin, (uint64_t)c.nouter, (uint64_t)ncomp};
    const uint64_t strides[3] = {(uint64_t)c.in_lstr * es, outer_bytes,
                                 ncomp > 1 ? (uint64_t)c.in_cstr * es : outer_bytes * (uint64_t)c.nouter};
    const uint32_t box[4] = {(uint32_t)(tx * u), (uint32_t)std::min(256, c.nin), 1, 1};
    make_prefetch(c.pf, c.in, dims, strides, box, (c.nin + 255) / 256, 256, PREFETCH_DIST);
}

void Solver::row_prefetch(RowArgs& r, bool f64, bool c2r, int L, int ncomp) const {
    const int elem = c2r ? (f64 ? 16 : 8) : (r.in_f64 ? 8 : 4);
    const uint64_t row_bytes = (uint64_t)r.nin * elem;
    if ((double)row_bytes * r.nrows * ncomp < PREFETCH_MIN_BYTES) return;
    const uint64_t units = (row_bytes + 7) / 8;
    const int tr = fast_row_tile_rows(f64 ? 1 : 0, L);
    const uint64_t n2 = (uint64_t)(r.nrows / r.n1);
    const uint64_t s2 = (uint64_t)r.in_s2 * elem;
    const uint64_t dims[4] = {units, (uint64_t)r.n1, n2, (uint64_t)ncomp};
    const uint64_t strides[3] = {(uint64_t)r.in_s1 * elem, s2, ncomp > 1 ? (uint64_t)r.in_cstr * elem : s2 * n2};
    const uint32_t box[4] = {(uint32_t)std::min<uint64_t>(256, (units + 1) / 2 * 2), (uint32_t)std::min(tr, r.n1), 1, 1};
    make_prefetch(r.pf, r.in, dims, strides, box, (int)((units + 255) / 256), 256, PREFETCH_DIST);
}

// the ROT rows run two CTAs per SM: the block one wave of resident blocks
// ahead starts as this one ends, so its rows are fetched into L2 meanwhile
#ifndef FLB_ROWROT_PREFETCH
#define FLB_ROWROT_PREFETCH 1
#endif
void Solver::rowrot_prefetch(RowFusedArgs& f, bool f64, int L, int ncomp) const {
    const int rows = fast_rowrot_rows(f64 ? 1 : 0, L);
    const uint64_t elem = f64 ? 16 : 8;
    const uint64_t row_bytes = (uint64_t)f.nin * elem;
    if (!FLB_ROWROT_PREFETCH || rows == 0 || (double)row_bytes * f.n1 * f.n2 * ncomp < PREFETCH_MIN_BYTES) return;
    const uint64_t units = (row_bytes + 7) / 8;
    const uint64_t n2 = (uint64_t)f.n2;
    const uint64_t s2 = (uint64_t)f.s2 * elem;
    const uint64_t dims[4] = {units, (uint64_t)f.n1, n2, (uint64_t)ncomp};
    const uint64_t strides[3] = {(uint64_t)f.s1 * elem, s2, ncomp > 1 ? (uint64_t)f.cstr * elem : s2 * n2};
    const uint32_t box[4] = {(uint32_t)std::min<uint64_t>(256, (units + 1) / 2 * 2), (uint32_t)std::min(rows, f.n1), 1, 1};
    make_prefetch(f.pf, f.in, dims, strides, box, (int)((units + 255) / 256), 256, 2 * 148);
}

const void* Solver::stage_table(int n, bool f64, int r1) {
    if (r1 == 0) r1 = fast_radix1(f64 ? 1 : 0, n);
    const int64_t key = ((int64_t)1 << 40) + ((int64_t)r1 << 32) + (int64_t)n * 2 + (f64 ? 1 : 0);
    auto it = twiddles.find(key);
    if (it != twiddles.end()) return it->second;
    const int len = fast_stage_table_len_r1(n, r1);
    std::vector<double> w(2 * (size_t)std::max(len, 1), 0.0);
    for (int e = 0; e < len; ++e) {
        int q = 0, M = 1;
        fast_stage_exponent(n, r1, e, &q, &M);
        const long double a = -2.0L * (long double)M_PI * (long double)q / (long double)M;
        w[2 * e] = (double)cosl(a);
        w[2 * e + 1] = (double)sinl(a);
    }
    void* d = nullptr;
    if (f64) {
        check_cuda(cudaMalloc(&d, w.size() * sizeof(double)), "twiddle allocation");
        check_cuda(cudaMemcpy(d, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice), "twiddle upload");
    } else {
        std::vector<float> wf(w.size());
        for (size_t i = 0; i < w.size(); ++i) wf[i] = (float)w[i];
        check_cuda(cudaMalloc(&d, wf.size() * sizeof(float)), "twiddle allocation");
        check_cuda(cudaMemcpy(d, wf.data(), wf.size() * sizeof(float), cudaMemcpyHostToDevice), "twiddle upload");
    }
    twiddles[key] = d;
    return d;
}

const void* Solver::twiddle_plain(int L, bool f64) {
    const int64_t key = -((int64_t)L * 2 + (f64 ? 1 : 0));
    auto it = twiddles.find(key);
    if (it != twiddles.end()) return it->second;
    std::vector<double> w(2 * (size_t)L);
    for (int q = 0; q < L; ++q) {
        const long double a = -2.0L * (long double)M_PI * (long double)q / (long double)L;
        w[2 * q] = (double)cosl(a);
        w[2 * q + 1] = (double)sinl(a);
    }
    void* d = nullptr;
    if (f64) {
        check_cuda(cudaMalloc(&d, w.size() * sizeof(double)), "twiddle allocation");
        check_cuda(cudaMemcpy(d, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice), "twiddle upload");
    } else {
        std::vector<float> wf(w.size());
        for (size_t i = 0; i < w.size(); ++i) wf[i] = (float)w[i];
        check_cuda(cudaMalloc(&d, wf.size() * sizeof(float)), "twiddle allocation");
        check_cuda(cudaMemcpy(d, wf.data(), wf.size() * sizeof(float), cudaMemcpyHostToDevice), "twiddle upload");
    }
    twiddles[key] = d;
    return d;
}

// Restrict a pass to the slab [slab_lo, slab_hi) of dimension slab_dim (not
// its line axis): both arrays start at the slab, the lines outside it are skipped.
void Solver::restrict_slab(PassArgs& A, bool in_f64, bool out_f64) const {
    const int a = (A.axis == 0) ? 1 : 0;
    const int d = slab_dim;
    const int64_t lo = slab_lo;
    if (A.fused) {
        // the folded Green's function is not folded along d: shift it with the slab
        A.mult.green = (const char*)A.mult.green + lo * A.mult.gstr[d] * (precision == 64 ? 8 : 4);
    }
    const int64_t ein = (in_f64 ? 8 : 4) * (A.st[0].in_cplx ? 2 : 1);
    const int64_t eout = (out_f64 ? 8 : 4) * (A.st[A.fused ? 1 : 0].out_cplx ? 2 : 1);
    A.in = (const char*)A.in + lo * A.in_str[d] * ein;
    A.out = (char*)A.out + lo * A.out_str[d] * eout;
    if (d == a) A.n_a = slab_hi - slab_lo;
    else A.n_b = slab_hi - slab_lo;
    A.nlines = (int64_t)A.n_a * A.n_b;
}

void Solver::run_pass(const PassArgs& Ain, bool f64, bool in_f64, bool out_f64, const char* name) {
    PassArgs A = Ain;
    if (slab_dim >= 0 && A.axis != slab_dim && (!A.fused || (A.mult.mode == 1 && A.mult.gfold[slab_dim] == 0)))
        restrict_slab(A, in_f64, out_f64);
    const int fk = fast_kind(A, f64, in_f64, out_f64);
    if (dry) {
        dry_passes.push_back(A);
        dry_flags.push_back((f64 ? 1 : 0) | (in_f64 ? 2 : 0) | (out_f64 ? 4 : 0));
        dry_names.push_back(name);
        dry_fast.push_back(fk);
        return;
    }
    // a connected share's y passes must reach the owners' column arrays
    FLB_CHECK(!(peers.n > 0 && owned() && slab_dim == 2 && A.axis == 1 && !A.fused) || (fk == 1 && A.ncomp == 1),
              "a share connected to its peers' column arrays needs register-DFT y passes");
    for (int s2 = 0; s2 <= A.fused; ++s2)
        if (!A.st[s2].tw) A.st[s2].tw = twiddle(A.st[s2].M, f64);
    // algorithmic bytes: source and kept output lines once, the folded Green's spectrum once
    const int64_t nc = A.ncomp;
    const double es = f64 ? 8.0 : 4.0;
    const LineStage& last = A.st[A.fused ? 1 : 0];
    double bytes = (double)A.n_src * A.nlines * nc * (A.st[0].in_cplx ? 2 : 1) * (in_f64 ? 8.0 : 4.0) +
                   (double)last.n_store * A.nlines * nc * (last.out_cplx ? 2 : 1) * (out_f64 ? 8.0 : 4.0);
    if (A.fused) bytes += (double)gfold_n[0] * gfold_n[1] * gfold_n[2] * es;
    const int k = timed_begin(name, bytes);
    if (fk) launch_fast(A, fk, f64, in_f64, out_f64);
    else check_cuda(launch_line_pass(A, f64 ? 1 : 0, in_f64 ? 1 : 0, out_f64 ? 1 : 0, stream), "line pass launch");
    timed_end(k);
}

int Solver::timed_begin(const char* name, double bytes) {
    const int k = pass_idx++;
    if (!timing) return k;
    if ((int)pass_ms.size() <= k) {
        pass_ms.resize(k + 1, 0.0);
        pass_bytes.resize(k + 1, 0.0);
        pass_calls.resize(k + 1, 0);
        pass_names.resize(k + 1);
    }
    pass_bytes[k] = bytes;
    pass_names[k] = name;
    while ((int)ev.size() < 2 * (k + 1)) {
        cudaEvent_t e;
        check_cuda(cudaEventCreate(&e), "event");
        ev.push_back(e);
    }
    cudaEventRecord(ev[2 * k], stream);
    return k;
}

void Solver::timed_end(int k) {
    if (timing) cudaEventRecord(ev[2 * k + 1], stream);
}

void Solver::collect_timing() {
    if (!timing) return;
    check_cuda(cudaEventSynchronize(ev[2 * (pass_idx - 1) + 1]), "timing");
    for (int k = 0; k < pass_idx; ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]);
        pass_ms[k] += ms;
        pass_calls[k] += 1;
    }
}

// ---------------------------------------------------------------- Green
void Solver::compute_green() {
    // Solver.cpp:980-1106
    const int kind = green_type;
    double length = alpha * h[0];
    if (kind == HEJ_0) length = h[0] / M_PI;
    const bool iso_kernel = (kind == HEJ_2 || kind == HEJ_4 || kind == HEJ_6 || kind == HEJ_8 || kind == HEJ_10 || kind == HEJ_0 ||
                             kind == LGF_2);
    FLB_CHECK(!(iso_kernel && ((ndim == 3 && (h[0] != h[1] || h[1] != h[2])) || (ndim == 2 && h[0] != h[1]))),
              "You are trying to use a regularized kernel or a LGF while not having dx=dy=dz.");
    const bool is_hej = (kind == HEJ_2 || kind == HEJ_4 || kind == HEJ_6 || kind == HEJ_8 || kind == HEJ_10);
    const bool is_lgf = (kind == LGF_2 || kind == LGF_4 || kind == LGF_6 || kind == LGF_8);
    const bool is_meh = (kind == MEHR_4L || kind == MEHR_4F || kind == MEHR_6L || kind == MEHR_6F);

    bool spec[3] = {false, false, false};
    double symstart[3] = {0, 0, 0}, hfact[3] = {0, 0, 0}, kfact[3] = {0, 0, 0}, koffset[3] = {0, 0, 0};
    for (int ip = 0; ip < ndim; ++ip) {
        const DirPlan& p = grn[ip];
        const int d = p.dim;
        spec[d] = p.is_spectral;
        symstart[d] = p.symstart;
        hfact[d] = h[d];
        if (p.is_spectral) {
            hfact[d] = 0.0;
            kfact[d] = p.kfact;
            koffset[d] = p.koffset;
        }
        if (p.type == EMPTY) hfact[d] = 0.0;
    }
    int nspec = 0;
    for (int d = 0; d < ndim; ++d)
        if (spec[d]) ++nspec;
    const int nunb = ndim - nspec;

    // spectral extents of the Green's function and its topology 0 (Solver.cpp:727-781)
    int spec_n[3] = {topo_phys->nglob[0], topo_phys->nglob[1], topo_phys->nglob[2]};
    bool spec_cplx = false;
    for (int ip = 0; ip < ndim; ++ip) {
        spec_n[grn[ip].dim] = grn[ip].n_out;
        spec_cplx = spec_cplx || grn[ip].isr2c;
    }
    int size0[3] = {spec_n[0], spec_n[1], spec_n[2]};
    bool cplx0 = spec_cplx;
    for (int ip = ndim - 1; ip >= 0; --ip)
        if (grn[ip].isr2c_done_by_fft()) {
            size0[grn[ip].dim] *= 2;
            cplx0 = false;
        }
    const size_t n0 = (size_t)size0[0] * size0[1] * size0[2] * (cplx0 ? 2 : 1);
    const size_t ns = (size_t)spec_n[0] * spec_n[1] * spec_n[2] * (spec_cplx ? 2 : 1);
    size_t nmax = std::max(n0, ns);
    // intermediate states are never larger than max(start, end) along each transformed direction
    double* gb[2] = {nullptr, nullptr};
    if (!dry) {
        // every intermediate state holds at most nmax doubles (each pass keeps or halves/doubles
        // the real count of one direction between the two ends)
        check_cuda(cudaMalloc(&gb[0], nmax * sizeof(double)), "Green buffer");
        check_cuda(cudaMalloc(&gb[1], nmax * sizeof(double)), "Green buffer");
    }

    GreenEvalArgs E;
    memset(&E, 0, sizeof(E));
    E.kind = kind;
    E.nunb = nunb;
    for (int d = 0; d < 3; ++d) {
        E.size[d] = size0[d];
        E.symstart[d] = symstart[d];
        E.hfact[d] = hfact[d];
        E.kfact[d] = kfact[d];
        E.koffset[d] = koffset[d];
    }
    E.cplx = cplx0;
    const int ax0 = grn[0].dim;
    E.ax[0] = ax0;
    E.ax[1] = (ax0 + 1) % 3;
    E.ax[2] = (ax0 + 2) % 3;
    E.length = length;
    std::vector<double> table;
    std::vector<FarTerm> far;
    double far_log = 0.0;
    double* d_table = nullptr;
    FarTerm* d_far = nullptr;
    if (nunb == 3) {
        E.hgrid = hfact[E.ax[0]];
        if (is_lgf || is_meh) {
            E.tableN = load_lgf_table(kind, 3, table);
            farfield_terms(kind, 3, far, far_log);
        } else {
            E.set_g0 = 1;
            const double s3 = std::sqrt(M_PI * M_PI * M_PI);
            const double r2 = std::sqrt(2.0);
            switch (kind) {
                case HEJ_2: E.g0 = -r2 / (4.0 * length * s3); break;
                case HEJ_4: E.g0 = -3.0 * r2 / (8.0 * length * s3); break;
                case HEJ_6: E.g0 = -15.0 * r2 / (32.0 * length * s3); break;
                case HEJ_8: E.g0 = -35.0 * r2 / (64.0 * length * s3); break;
                case HEJ_10: E.g0 = -315.0 * r2 / (512.0 * length * s3); break;
                case HEJ_0: E.g0 = -1.0 / (2.0 * M_PI * M_PI * length); break;
                case CHAT_2: {
                    const double hp = hfact[0] * hfact[1] * hfact[2];
                    E.g0 = -0.5 * std::pow(1.5 * (1.0 / (2.0 * M_PI)) * hp, 2. / 3.) / hp;
                    break;
                }
                default: FLB_CHECK(false, "Green Function type unknown.");
            }
        }
    } else if (nunb == 2) {
        const double ha = hfact[E.ax[0]], hb = hfact[E.ax[1]], hc = hfact[E.ax[2]];
        E.r_eq2d = (1.0 / std::sqrt(M_PI)) * std::sqrt(ha * hb + hb * hc + hc * ha);
        E.r_cut = (ha + hb + hc) * .2;
        E.k_cut = (kfact[E.ax[0]] + kfact[E.ax[1]] + kfact[E.ax[2]]) * 0.2;
        E.chat2d_origin = (kind == CHAT_2);
        if (is_lgf || is_meh) {
            E.tableN = load_lgf_table(kind, 2, table);
            farfield_terms(kind, 2, far, far_log);
        }
    } else if (nunb == 1) {
        FLB_CHECK(kind != HEJ_0, "HEJ0 kernel not available for 1D unbounded problems.");
        E.k_cut = (kfact[E.ax[0]] + kfact[E.ax[1]] + kfact[E.ax[2]]) * 0.2;
        E.hgrid = hfact[E.ax[0]] + hfact[E.ax[1]] + hfact[E.ax[2]];
    } else {
        E.hgrid = h[0];
        E.set_g0 = (koffset[0] + koffset[1] + koffset[2] < 0.2);
    }
    if (!table.empty() && !dry) {
        check_cuda(cudaMalloc(&d_table, table.size() * sizeof(double)), "LGF table");
        check_cuda(cudaMemcpy(d_table, table.data(), table.size() * sizeof(double), cudaMemcpyHostToDevice), "LGF table");
        E.table = d_table;
    }
    if (!far.empty() && !dry) {
        check_cuda(cudaMalloc(&d_far, far.size() * sizeof(FarTerm)), "far field");
        check_cuda(cudaMemcpy(d_far, far.data(), far.size() * sizeof(FarTerm), cudaMemcpyHostToDevice), "far field");
        E.far = d_far;
        E.nfar = (int)far.size();
        E.far_log = far_log;
    }
    E.out = gb[0];
    if (!dry) check_cuda(launch_green_eval(E, stream), "Green evaluation");

    // forward transforms of the Green's function (Solver.cpp:1058-1076), FP64
    ArrState cur;
    for (int d = 0; d < 3; ++d) cur.n[d] = size0[d];
    cur.cplx = cplx0;
    int cb = 0;
    for (int ip = 0; ip < ndim; ++ip) {
        const DirPlan& p = grn[ip];
        if (spec[p.dim]) continue;
        // a real-to-real transform of complex storage acts on the real part only (the reference's
        // r2r plan with stride nf = 2, src/FFTW_plan_dim.cpp:323-331); the imaginary part is zero here
        ArrState nxt = cur;
        nxt.n[p.dim] = p.n_out;
        nxt.cplx = cur.cplx || p.isr2c;
        PassArgs A = base_pass(p.dim, cur, 1, 1);
        LineStage S;
        memset(&S, 0, sizeof(S));
        LineSpec& sp = S.spec[0];
        sp.kind = (p.type == MIXUNB) ? LK_DCT1 : (p.isr2c ? LK_R2C : LK_C2C);
        sp.sign = -1;
        sp.n_in = p.n_in[0];
        sp.fi = sp.fo = 0;
        sp.postpro = PP_NONE;
        S.spec[1] = S.spec[2] = sp;
        S.M = fft_length(sp.kind, sp.n_in);
        factorize(S.M, S);
        S.n_b = p.isr2c ? 2 * p.n_out : p.n_out;
        S.fieldstart = 0;
        S.n_o = p.n_out;
        S.in_cplx = cur.cplx;
        S.out_cplx = nxt.cplx;
        S.n_store = S.n_o;
        S.tw = nullptr;
        A.st[0] = S;
        set_strides_internal(A.in_str, A.in_cstr, cur, false);
        set_strides_internal(A.out_str, A.out_cstr, nxt, false);
        A.in = gb[cb];
        A.out = gb[1 - cb];
        fit_lines(A, sizeof(double));
        run_pass(A, true, true, true, "green");
        cb = 1 - cb;
        cur = nxt;
    }

    // folded layout of the working-precision copy
    for (int d = 0; d < 3; ++d) {
        gfold_M[d] = 0;
        gfold_n[d] = st[ndim].n[d];
    }
    for (int ip = 0; ip < ndim; ++ip) {
        const DirPlan& p = fwd[ip];
        if ((p.type == PERPER || p.type == UNBUNB) && !p.isr2c) {
            gfold_M[p.dim] = p.n_in[0];
            gfold_n[p.dim] = p.n_in[0] / 2 + 1;
        }
    }
    for (int d = 0; d < 3; ++d)
        FLB_CHECK(spec_n[d] == st[ndim].n[d], "Topo of Green has to be the same as Topo of field");
    if (has_xlast) {
        // the x-last order folds its complex-to-complex directions the same
        // way; its folded extents must be those of this array (they are for
        // every all-unbounded problem: 2N-point lines fold to N + 1 values,
        // the N + 1 of the real-to-complex direction need no fold)
        for (int d = 0; d < 3; ++d) xgfold_M[d] = 0;
        for (int ip = 0; ip < ndim; ++ip) {
            const DirPlan& p = xfwd[ip];
            const bool fold = (p.type == UNBUNB || p.type == PERPER) && !p.isr2c;
            const int fn = fold ? p.n_in[0] / 2 + 1 : xst[ndim].n[p.dim];
            if (fold) xgfold_M[p.dim] = p.n_in[0];
            if (fn != gfold_n[p.dim]) has_xlast = false;
        }
    }
    const bool f64 = (precision == 64);
    const int64_t gq = f64 ? 16 : 32;  // rows of the folded spectrum on 128-byte boundaries
    gstr[0] = 1;
    gstr[1] = ((int64_t)gfold_n[0] + gq - 1) / gq * gq;
    gstr[2] = gstr[1] * gfold_n[1];
    const size_t gsz = (size_t)gstr[2] * gfold_n[2];
    if (dry) return;
    if (green) cudaFree(green);
    check_cuda(cudaMalloc(&green, gsz * (f64 ? 8 : 4)), "Green spectrum");

    GreenFinalArgs F;
    memset(&F, 0, sizeof(F));
    F.spec = gb[cb];
    F.spec_cplx = cur.cplx;
    for (int d = 0; d < 3; ++d) {
        F.spec_n[d] = cur.n[d];
        F.fold_n[d] = gfold_n[d];
        F.fold_str[d] = gstr[d];
    }
    F.volfact = volfact;
    F.complete = (ndim == 3 && nspec == 1 && (is_hej || is_lgf || is_meh));
    if (F.complete) {
        for (int d = 0; d < 3; ++d)
            if (spec[d]) F.spec_dim = d;
    }
    F.kind = kind;
    for (int ip = 0; ip < 3; ++ip) F.kfact[grn[ip].dim] = grn[ip].kfact;
    for (int d = 0; d < 3; ++d) {
        F.koffset[d] = koffset[d];
        F.symstart[d] = symstart[d];
    }
    const int axl = grn[ndim - 1].dim;
    F.ax[0] = axl;
    F.ax[1] = (axl + 1) % 3;
    F.ax[2] = (axl + 2) % 3;
    F.hgrid = h[0];
    F.length = length;
    F.reset0 = (F.complete || nunb == 0) && (koffset[0] + koffset[1] + koffset[2] < 0.2);
    // the stored spectrum is normfact * volfact * G (dothemagic's normfact applied
    // once here instead of per solve)
    F.scale = normfact;
    F.out = green;
    F.out_f64 = f64;
    check_cuda(launch_green_final(F, stream), "Green finalisation");
    check_cuda(cudaStreamSynchronize(stream), "Green setup");
    cudaFree(gb[0]);
    cudaFree(gb[1]);
    if (d_table) cudaFree(d_table);
    if (d_far) cudaFree(d_far);
}

// ---------------------------------------------------------------- setup / solve
void Solver::setup() {
    cs_follows = false;
    FLB_CHECK(!is_setup, "setup was already called");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    FLB_CHECK(e == cudaSuccess && ndev > 0, "no CUDA device available (%s): this library has no CPU path",
              cudaGetErrorString(e));
    compute_green();
    if (owned()) slice_green();
    build_ksym();
    plan_xlast();
    ensure_buffers(1);
    is_setup = true;
}

// The curl symbols K_{d,c}(i) of a solver that can run ROT (three components
// and a derivative order), for the fused ROT column pass: 9 tables of the
// spectral extents, evaluated on the device with the functions of the
// pointwise multiply.
void Solver::build_ksym() {
    if (!have_diff || lda != 3 || dry || ksym) return;
    if (has_xlast && !xlast_active) {
        // the x-last order's tables first (its spectral extents and symmetries)
        swap_order();
        build_ksym();
        swap_order();
    }
    const MultSpec G = mult_spec(ROT);
    int n[3];
    kstr = 1;
    for (int d = 0; d < 3; ++d) {
        n[d] = st[ndim].n[d];
        kstr = std::max(kstr, n[d]);
    }
    const bool f64 = (precision == 64);
    check_cuda(cudaMalloc(&ksym, (size_t)9 * kstr * 2 * (f64 ? 8 : 4)), "curl symbol tables");
    check_cuda(launch_ksym_table(G, n, kstr, ksym, f64 ? 1 : 0, stream), "curl symbol tables");
    check_cuda(cudaStreamSynchronize(stream), "curl symbol tables");
}

// A solver set up for a share keeps only its columns [own[2], own[3]) of the
// folded Green's spectrum (x is not folded there), rows on 128-byte
// boundaries; `green` is placed where the full array would start, so the
// x-slab offset of the last-direction pass lands on the share.
void Solver::slice_green() {
    const bool f64 = (precision == 64);
    const size_t es = f64 ? 8 : 4;
    FLB_CHECK(gfold_M[0] == 0 && gstr[0] == 1 && own[3] <= gfold_n[0] && gstr[2] == gstr[1] * gfold_n[1],
              "the Green's spectrum cannot be split by columns");
    const int64_t gq = f64 ? 16 : 32;
    const int64_t w = own[3] - own[2], wp = (w + gq - 1) / gq * gq;
    void* gc = nullptr;
    check_cuda(cudaMalloc(&gc, (size_t)wp * gfold_n[1] * gfold_n[2] * es), "Green spectrum share");
    check_cuda(cudaMemcpy2D(gc, wp * es, (const char*)green + own[2] * es, gstr[1] * es, w * es,
                            (size_t)gfold_n[1] * gfold_n[2], cudaMemcpyDeviceToDevice),
               "Green spectrum share copy");
    cudaFree(green);
    green_share = gc;
    green = reinterpret_cast<void*>(reinterpret_cast<uintptr_t>(gc) - (uintptr_t)own[2] * es);
    gstr[1] = wp;
    gstr[2] = wp * gfold_n[1];
}

void Solver::ensure_buffers(int nbatch) {
    const bool f64 = (precision == 64);
    const size_t es = f64 ? 8 : 4;
    if (owned()) {
        // one rank's share: the planes it owns, and its spectrum columns over every plane
        FLB_CHECK(nbatch == 1, "a solver set up for a share of the planes solves one field at a time");
        const ArrState& sp = st[ndim - 1];
        const size_t xneed = (size_t)xpitch * sp.n[1] * sp.n[2] * 2;
        if (!xbuf) check_cuda(cudaMalloc(&xbuf, xneed * es), "column work buffer");
    }
    for (int b = 0; b < 2; ++b) {
        const size_t need = work_reals(b, nbatch);
        if (need > buf_elems[b]) {
            drop_graphs();  // captured solves point at the old arrays
            if (buf[b]) cudaFree(buf[b]);
            buf[b] = nullptr;
            check_cuda(cudaMalloc(&buf[b], need * es), "work buffer");
            buf_elems[b] = need;
        }
    }
    buf_batch = std::max(buf_batch, nbatch);
}

// Captured solves (flups_solve_graph, and the group graphs that count on
// `gen`) point at the work arrays and follow the switches in force when they
// were captured: reallocation and switch changes drop them.
void Solver::drop_graphs() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
    ++gen;
}

size_t Solver::device_bytes(int nbatch) const {
    const size_t es = (precision == 64) ? 8 : 4;
    size_t total = 0;
    for (int b = 0; b < 2; ++b) total += work_reals(b, nbatch) * es;
    if (owned()) total += (size_t)xpitch * st[ndim - 1].n[1] * st[ndim - 1].n[2] * 2 * es;
    // (a share holds its columns of the Green's spectrum: gstr describes that array after set-up)
    total += (size_t)gstr[2] * gfold_n[2] * es;
    if (ksym) total += (size_t)9 * kstr * 2 * es;
    if (xksym) total += (size_t)9 * xkstr * 2 * es;
    return total;
}

static bool is_device_ptr(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

void Solver::do_fft_forward(const double* user_in, int nbatch) {
    for (int ip = 0; ip < ndim - 1; ++ip) fwd_pass(ip, user_in, nbatch);
}

void Solver::fwd_pass(int ip, const double* user_in, int nbatch) {
    const bool f64 = (precision == 64);
    const int es = f64 ? 8 : 4;
    const DirPlan& p = fwd[ip];
    PassArgs A = base_pass(p.dim, st[ip], lda * nbatch, lda);
    A.st[0] = stage_forward(p, ip, f64);
    if (ip == 0) {
        set_strides_user(A.in_str, A.in_cstr);
        A.in = user_in;
    } else {
        set_strides_internal(A.in_str, A.in_cstr, st[ip]);
        A.in = work_base((ip - 1) % 2);
    }
    set_strides_internal(A.out_str, A.out_cstr, st[ip + 1]);
    A.out = work_base(ip % 2);
    fit_lines(A, es);
    static const char* fn[3] = {"fwd0", "fwd1", "fwd2"};
    run_pass(A, f64, ip == 0 ? true : f64, f64, fn[ip]);
}

void Solver::do_fft_backward_fused(double* user_out, int type, int nbatch) {
    do_fused(type, nbatch);
    do_backward(user_out, type, nbatch);
}

void Solver::do_fused(int type, int nbatch) {
    const bool f64 = (precision == 64);
    const int es = f64 ? 8 : 4;
    const int ipl = ndim - 1;
    {
        // fused: forward ndim-1, multiply, backward ndim-1 (in place on state ndim-1)
        const DirPlan& p = fwd[ipl];
        const DirPlan& pb = (type == ROT) ? dif[ipl] : bwd[ipl];
        const bool rot = (type == ROT);
        PassArgs A = base_pass(p.dim, st[ipl], lda * nbatch, lda);
        A.fused = 1;
        A.comps_together = rot ? 1 : 0;
        if (rot) A.ncomp = 3;
        A.st[0] = stage_forward(p, ipl, f64);
        A.st[1] = stage_backward(pb, p, ipl, f64);
        A.mult = mult_spec(type);
        set_strides_internal(A.in_str, A.in_cstr, st[ipl]);
        set_strides_internal(A.out_str, A.out_cstr, st[ipl]);
        A.in = buf[(ipl - 1) % 2];
        A.out = buf[(ipl - 1) % 2];
        if (owned()) {
            // the rank's columns over every plane, column own[2] first (the
            // slab restriction along x adds own[2] columns back)
            const ArrState& sp = st[ipl];
            const int64_t str[3] = {1, xpitch, xpitch * sp.n[1]};
            for (int d = 0; d < 3; ++d) A.in_str[d] = A.out_str[d] = str[d];
            A.in_cstr = A.out_cstr = xpitch * sp.n[1] * sp.n[2];
            const uintptr_t base = reinterpret_cast<uintptr_t>(xbuf) - (uintptr_t)own[2] * (uintptr_t)(2 * es);
            A.in = reinterpret_cast<const void*>(base);
            A.out = reinterpret_cast<void*>(base);
        }
        fit_lines(A, es);
        if (rot && nbatch > 1) {
            const int64_t per = A.in_cstr * 3 * (st[ipl].cplx ? 2 : 1);
            for (int b = 0; b < nbatch; ++b) {
                PassArgs B = A;
                B.in = (const char*)A.in + (size_t)b * per * es;
                B.out = (char*)A.out + (size_t)b * per * es;
                run_pass(B, f64, f64, f64, "fused");
            }
        } else {
            run_pass(A, f64, f64, f64, "fused");
        }
    }
}

void Solver::do_backward(double* user_out, int type, int nbatch) {
    for (int ip = ndim - 2; ip >= 0; --ip) bwd_pass(ip, user_out, type, nbatch);
}

void Solver::bwd_pass(int ip, double* user_out, int type, int nbatch) {
    const bool f64 = (precision == 64);
    const int es = f64 ? 8 : 4;
    const DirPlan& p = (type == ROT) ? dif[ip] : bwd[ip];
    PassArgs A = base_pass(fwd[ip].dim, st[ip + 1], lda * nbatch, lda);
    A.st[0] = stage_backward(p, fwd[ip], ip, f64);
    set_strides_internal(A.in_str, A.in_cstr, st[ip + 1]);
    A.in = work_base(ip % 2);
    if (ip == 0) {
        set_strides_user(A.out_str, A.out_cstr);
        A.out = user_out;
    } else {
        set_strides_internal(A.out_str, A.out_cstr, st[ip]);
        A.out = work_base((ip - 1) % 2);
    }
    fit_lines(A, es);
    static const char* bn[3] = {"bwd0", "bwd1", "bwd2"};
    run_pass(A, f64, f64, ip == 0 ? true : f64, bn[ip]);
}

// Overlapped middle passes (STD, x transformed first, device arrays): after
// the x pass, the y forward, fused z and y inverse passes of an x-slab only
// touch that slab, so slab k's fused pass (issue-bound) runs on one stream
// while slab k+1's y forward and slab k-1's y inverse (memory-bound) run on
// others; the x inverse pass waits for every slab.
bool Solver::overlap_ok(int type) const {
    return overlap && !timing && !dry && !capturing && ndim == 3 && type == STD && fwd[0].dim == 0 && slab_dim < 0 &&
           gfold_M[0] == 0 && st[1].n[0] >= 64;
}

void Solver::solve_overlap(const double* din, double* dout, int type, int nbatch) {
    if (!ov_stream[0]) {
        for (int i = 0; i < 2; ++i) check_cuda(cudaStreamCreateWithFlags(&ov_stream[i], cudaStreamNonBlocking), "stream");
        check_cuda(cudaEventCreateWithFlags(&ov_ev0, cudaEventDisableTiming), "event");
        for (int k = 0; k < kOvSlabs; ++k) {
            check_cuda(cudaEventCreateWithFlags(&ov_evf[k], cudaEventDisableTiming), "event");
            check_cuda(cudaEventCreateWithFlags(&ov_evg[k], cudaEventDisableTiming), "event");
        }
    }
    pass_idx = 0;
    fwd_pass(0, din, nbatch);
    check_cuda(cudaEventRecord(ov_ev0, stream), "event record");
    const cudaStream_t main = stream;
    const int nx = st[1].n[0];
    // slab bounds on 32-column boundaries (whole CTA tiles, 128-byte Green rows)
    const int chunks = (nx + 31) / 32;
    const int ns = std::min(kOvSlabs, chunks);
    for (int k = 0; k < ns; ++k) {
        const int lo = std::min(nx, (int)((int64_t)k * chunks / ns) * 32);
        const int hi = (k == ns - 1) ? nx : std::min(nx, (int)((int64_t)(k + 1) * chunks / ns) * 32);
        slab_dim = 0;
        slab_lo = lo;
        slab_hi = hi;
        stream = ov_stream[0];
        if (k == 0) check_cuda(cudaStreamWaitEvent(stream, ov_ev0, 0), "stream wait");
        fwd_pass(1, nullptr, nbatch);
        check_cuda(cudaEventRecord(ov_evf[k], stream), "event record");
        stream = ov_stream[1];
        check_cuda(cudaStreamWaitEvent(stream, ov_evf[k], 0), "stream wait");
        do_fused(type, nbatch);
        check_cuda(cudaEventRecord(ov_evg[k], stream), "event record");
        stream = main;
        check_cuda(cudaStreamWaitEvent(stream, ov_evg[k], 0), "stream wait");
        bwd_pass(1, nullptr, type, nbatch);
    }
    slab_dim = -1;
    stream = main;
    bwd_pass(0, dout, type, nbatch);
}

void Solver::solve(double* field, double* rhs, int type, int nbatch) {
    FLB_CHECK(is_setup, "flups_setup must be called before flups_solve");
    FLB_CHECK((type == ROT && lda == 3) || (type != ROT), "You need vectors when using the ROT solver");
    FLB_CHECK(!(type == ROT && odiff == NOD), "If calling the ROT solver, you need to initialize it with orderDiff = SPE or orderDiff = FD2");
    FLB_CHECK((type == ROT && (odiff == SPE || odiff == FD2 || odiff == FD4 || odiff == FD6)) || (type != ROT),
              "The differenciation order asked does not exist ");
    FLB_CHECK(field != nullptr, "field is NULL");
    FLB_CHECK(rhs != nullptr, "rhs is NULL");
    FLB_CHECK(nbatch >= 1, "nbatch must be >= 1");
    FLB_CHECK(!owned(), "this solver holds one rank's share of the planes: use the flups_b200_slab_* steps");
    const bool follows = cs_follows;
    cs_follows = false;
    ensure_buffers(nbatch);
    if (autotune) autotune_passes(type, nbatch);
    const size_t user_elems = topo_phys->memsize() * (size_t)nbatch;
    // (a solve being captured has device arrays, checked before the capture)
    const bool dev_in = capturing || is_device_ptr(rhs), dev_out = capturing || is_device_ptr(field);
    if ((!dev_in || !dev_out) && streamed_ok()) {
        solve_streamed(field, rhs, !dev_in, !dev_out, type, nbatch, follows);
        return;
    }
    double* din = rhs;
    double* dout = field;
    if (!dev_in || !dev_out) {
        if (stage_elems < user_elems) {
            if (stage_in) cudaFree(stage_in);
            check_cuda(cudaMalloc(&stage_in, user_elems * sizeof(double)), "staging buffer");
            stage_elems = user_elems;
        }
    }
    if (!dev_in) {
        check_cuda(cudaMemcpyAsync(stage_in, rhs, user_elems * sizeof(double), cudaMemcpyHostToDevice, stream), "rhs upload");
        din = stage_in;
    }
    if (!dev_out) dout = stage_in;
    pass_idx = 0;
    if (dev_in && dev_out && overlap_ok(type)) {
        solve_overlap(din, dout, type, nbatch);
    } else {
        const bool xl = xlast_ok(type);
        if (xl) swap_order();
        do_fft_forward(din, nbatch);
        do_fft_backward_fused(dout, type, nbatch);
        if (xl) swap_order();
    }
    collect_timing();
    if (!dev_out) {
        check_cuda(cudaMemcpyAsync(field, dout, user_elems * sizeof(double), cudaMemcpyDeviceToHost, stream), "field download");
    }
    if (!async || !dev_out || !dev_in) check_cuda(cudaStreamSynchronize(stream), "solve");
    else check_cuda(cudaGetLastError(), "solve");
}

// ---------------------------------------------------------------- host arrays, streamed
// The passes before and after the fused one work on lines of the other two
// directions, so slabs of the last forward direction are independent there:
// slab k of rhs is uploaded while slab k-1 is transformed, and slab k of the
// result is downloaded while slab k+1 is transformed back.  Uploads and
// downloads use their own streams and staging arrays, so with async the
// upload of the next solve overlaps the download of this one.
bool Solver::streamed_ok() const {
    // slabs along z are contiguous in the user layout (x fastest)
    return !timing && ndim == 3 && fwd[ndim - 1].dim == 2 && st[0].n[2] >= 2;
}

void Solver::solve_streamed(double* field, double* rhs, bool in_host, bool out_host, int type, int nbatch, bool follows) {
    const int d = 2;
    const int nd = st[0].n[d];
    const int ns = std::min(kSlabs, nd);
    const size_t user_elems = topo_phys->memsize() * (size_t)nbatch;
    if (in_host && stage_elems < user_elems) {
        if (stage_in) cudaFree(stage_in);
        stage_in = nullptr;
        check_cuda(cudaMalloc(&stage_in, user_elems * sizeof(double)), "staging buffer");
        stage_elems = user_elems;
    }
    if (out_host && stage_out_elems < user_elems) {
        if (stage_out) cudaFree(stage_out);
        stage_out = nullptr;
        check_cuda(cudaMalloc(&stage_out, user_elems * sizeof(double)), "staging buffer");
        stage_out_elems = user_elems;
    }
    if (!h2d_stream) {
        check_cuda(cudaStreamCreateWithFlags(&h2d_stream, cudaStreamNonBlocking), "copy stream");
        check_cuda(cudaStreamCreateWithFlags(&d2h_stream, cudaStreamNonBlocking), "copy stream");
        for (int k = 0; k < kSlabs; ++k) {
            check_cuda(cudaEventCreateWithFlags(&ev_in[k], cudaEventDisableTiming), "event");
            check_cuda(cudaEventCreateWithFlags(&ev_fwd[k], cudaEventDisableTiming), "event");
            check_cuda(cudaEventCreateWithFlags(&ev_bwd[k], cudaEventDisableTiming), "event");
            check_cuda(cudaEventCreateWithFlags(&ev_out[k], cudaEventDisableTiming), "event");
        }
    }
    // async solves of host arrays in and out: the passes on cstream, which
    // follows the caller's stream unless this solver's last work was such a
    // solve (then the caller's stream ends in that solve's download wait, which
    // the passes need not wait for: back-to-back solves overlap one's download
    // with the next one's passes, and the copy engines never idle)
    const cudaStream_t caller = stream;
    const bool own = async && in_host && out_host && !capturing;
    if (own) {
        if (!cstream) {
            check_cuda(cudaStreamCreateWithFlags(&cstream, cudaStreamNonBlocking), "pass stream");
            check_cuda(cudaEventCreateWithFlags(&ev_entry, cudaEventDisableTiming), "event");
        }
        if (!follows) {
            check_cuda(cudaEventRecord(ev_entry, caller), "event record");
            check_cuda(cudaStreamWaitEvent(cstream, ev_entry, 0), "stream wait");
        }
        stream = cstream;
    }
    struct Restore {
        cudaStream_t& s;
        cudaStream_t keep;
        ~Restore() { s = keep; }
    } restore{stream, caller};
    int64_t ustr[3], ucstr;
    set_strides_user(ustr, ucstr);
    const int ncomp = lda * nbatch;
    double* din = in_host ? stage_in : rhs;
    double* dout = out_host ? stage_out : field;
    // an rhs that an earlier solve's download writes (a chain of async solves,
    // in place or field -> rhs): each slab's upload waits for that slab's
    // download when the arrays coincide, the first upload for all of them when
    // they only overlap
    const char* r_lo = reinterpret_cast<const char*>(rhs);
    const char* r_hi = r_lo + user_elems * sizeof(double);
    const bool after_dl = in_host && dl_lo && r_lo < dl_hi && dl_lo < r_hi;
    const bool per_slab = after_dl && r_lo == dl_lo;
    if (after_dl && !per_slab) check_cuda(cudaStreamWaitEvent(h2d_stream, ev_out[ns - 1], 0), "stream wait");
    pass_idx = 0;
    for (int k = 0; k < ns; ++k) {
        const int lo = (int)((int64_t)k * nd / ns), hi = (int)((int64_t)(k + 1) * nd / ns);
        if (in_host) {
            // the previous solve's passes have read this slab of the staging array
            check_cuda(cudaStreamWaitEvent(h2d_stream, ev_fwd[k], 0), "stream wait");
            if (per_slab) check_cuda(cudaStreamWaitEvent(h2d_stream, ev_out[k], 0), "stream wait");
            for (int c = 0; c < ncomp; ++c) {
                const size_t off = (size_t)c * ucstr + (size_t)lo * ustr[d];
                check_cuda(cudaMemcpyAsync(stage_in + off, rhs + off, (size_t)(hi - lo) * ustr[d] * sizeof(double),
                                           cudaMemcpyHostToDevice, h2d_stream),
                           "rhs upload");
            }
            check_cuda(cudaEventRecord(ev_in[k], h2d_stream), "event record");
            check_cuda(cudaStreamWaitEvent(stream, ev_in[k], 0), "stream wait");
        }
        slab_dim = d;
        slab_lo = lo;
        slab_hi = hi;
        do_fft_forward(din, nbatch);
        slab_dim = -1;
        check_cuda(cudaEventRecord(ev_fwd[k], stream), "event record");
    }
    do_fused(type, nbatch);
    for (int k = 0; k < ns; ++k) {
        const int lo = (int)((int64_t)k * nd / ns), hi = (int)((int64_t)(k + 1) * nd / ns);
        // the previous solve's download of this slab of the staging array is done
        if (out_host) check_cuda(cudaStreamWaitEvent(stream, ev_out[k], 0), "stream wait");
        slab_dim = d;
        slab_lo = lo;
        slab_hi = hi;
        do_backward(dout, type, nbatch);
        slab_dim = -1;
        if (out_host) {
            check_cuda(cudaEventRecord(ev_bwd[k], stream), "event record");
            check_cuda(cudaStreamWaitEvent(d2h_stream, ev_bwd[k], 0), "stream wait");
            for (int c = 0; c < ncomp; ++c) {
                const size_t off = (size_t)c * ucstr + (size_t)lo * ustr[d];
                check_cuda(cudaMemcpyAsync(field + off, stage_out + off, (size_t)(hi - lo) * ustr[d] * sizeof(double),
                                           cudaMemcpyDeviceToHost, d2h_stream),
                           "field download");
            }
            check_cuda(cudaEventRecord(ev_out[k], d2h_stream), "event record");
        }
    }
    stream = caller;
    if (out_host) {
        dl_lo = reinterpret_cast<const char*>(field);
        dl_hi = dl_lo + user_elems * sizeof(double);
    }
    // work queued later on the caller's stream sees the downloaded result (and,
    // through it, the passes)
    if (out_host) check_cuda(cudaStreamWaitEvent(stream, ev_out[ns - 1], 0), "stream wait");
    if (!async) check_cuda(cudaStreamSynchronize(stream), "solve");
    else check_cuda(cudaGetLastError(), "solve");
    cs_follows = own;
}

// ---------------------------------------------------------------- z-slab decomposition
// A solve split over ranks by planes of the last direction (the reference's
// pencil solve with its transposes, Solver.cpp:629-715 / SwitchTopoX_a2a.cpp):
// rank r owns user planes [z0, z1) and spectrum columns [x0, x1).  The x and
// y passes of its planes and the inverse ones only touch those planes; the
// last-direction pass needs every plane of its columns, so the spectrum is
// exchanged (all-to-all) before and after it.  Each step is the single-GPU
// pass restricted to a slab (slab_dim), so results equal the one-rank solve.
// The work arrays hold the rank's planes only (`work_base` places them where
// the full array would start, so the passes' slab offsets land on them) and
// `xbuf` holds its columns over every plane: a rank's memory falls with the
// rank count; the Green's spectrum is cut to its columns at set-up.  The
// user arrays of a step hold the rank's planes only (scalar field, lda 1).
int Solver::slab_check(int type) const {
    if (ndim != 3 || lda != 1 || type != STD) return -2;
    if (fwd[0].dim != 0 || fwd[1].dim != 1 || fwd[2].dim != 2) return -2;
    // the Green's spectrum is not folded along x, so a slab of columns reads its own part
    if (gfold_M[0] != 0) return -2;
    return 0;
}

int Solver::slab_own(int z0, int z1, int x0, int x1) {
    if (is_setup || owned()) return -1;
    if (int e = slab_check(STD); e) return e;
    if (z0 < 0 || z1 > st[0].n[2] || z0 >= z1 || x0 < 0 || x1 > st[ndim - 1].n[0] || x0 >= x1) return -2;
    own[0] = z0;
    own[1] = z1;
    own[2] = x0;
    own[3] = x1;
    const int64_t q = (precision == 64) ? 8 : 16;  // complex values per 128 bytes
    xpitch = (x1 - x0 + q - 1) / q * q;
    return 0;
}

// Every rank's column array, for y passes that store their outputs (and
// load their inputs) there directly: rank j owns columns [xs[j], xs[j+1]),
// its array has row pitch pitch[j]; this share's own entry must be its
// column array.  n = 0 goes back to the plane array and the exchanges.
int Solver::slab_peers(int n, void* const* cols, const int* xs, const int64_t* pitch) {
    if (!is_setup || !owned()) return -1;
    if (n == 0) {
        peers = flb::ColArgs::Peers{};
        return 0;
    }
    if (n < 1 || n > 8 || !cols || !xs || !pitch) return -2;
    if (xs[0] != 0 || xs[n] != st[ndim - 1].n[0]) return -2;
    int mine = -1;
    for (int j = 0; j < n; ++j) {
        if (xs[j + 1] <= xs[j] || pitch[j] < xs[j + 1] - xs[j] || !cols[j]) return -2;
        if (xs[j] == own[2] && xs[j + 1] == own[3]) mine = j;
    }
    if (mine < 0 || cols[mine] != xbuf || pitch[mine] != xpitch) return -2;
    // only the register-DFT column kernel stores to / loads from the owners'
    // arrays: a y pass that would run elsewhere (other line lengths, fast
    // kernels off) keeps the exchange steps
    if (!slab_y_fast()) return -2;
    flb::ColArgs::Peers P{};
    for (int j = 0; j < n; ++j) {
        P.col[j] = cols[j];
        P.xs[j] = xs[j];
        P.pitch[j] = pitch[j];
    }
    P.xs[n] = xs[n];
    P.n = n;
    peers = P;
    return 0;
}

// Whether the share's y forward and y inverse passes both run the register-DFT
// column kernel on one component (planned on the host, nothing launched).
bool Solver::slab_y_fast() {
    const bool keep = dry;
    const int keep_dim = slab_dim, keep_lo = slab_lo, keep_hi = slab_hi;
    dry = true;
    dry_passes.clear();
    dry_flags.clear();
    dry_names.clear();
    dry_fast.clear();
    slab_dim = 2;
    slab_lo = own[0];
    slab_hi = own[1];
    fwd_pass(1, nullptr, 1);
    bwd_pass(1, nullptr, STD, 1);
    bool ok = dry_fast.size() == 2;
    for (size_t i = 0; ok && i < dry_fast.size(); ++i) ok = dry_fast[i] == 1 && dry_passes[i].ncomp == 1 && dry_passes[i].axis == 1;
    dry_passes.clear();
    dry_flags.clear();
    dry_names.clear();
    dry_fast.clear();
    dry = keep;
    slab_dim = keep_dim;
    slab_lo = keep_lo;
    slab_hi = keep_hi;
    return ok;
}

// the array of buffer b seen from plane 0 (integer arithmetic: that base may
// precede the allocation; a pass restricted to the owned planes adds them back)
void* Solver::work_base(int b) const {
    if (!owned() || !buf[b]) return buf[b];
    const int k = b + 1;  // 3-D: buffer 0 holds state 1, buffer 1 state 2
    const int64_t plane = row_pitch(st[k]) * st[k].n[1] * (st[k].cplx ? 2 : 1) * (precision == 64 ? 8 : 4);
    return reinterpret_cast<void*>(reinterpret_cast<uintptr_t>(buf[b]) - (uintptr_t)((int64_t)own[0] * plane));
}

// the user array of the owned planes seen from plane 0 (integer arithmetic, as above)
static uintptr_t slab_base(const void* p, int z0, int64_t plane_elems) {
    return reinterpret_cast<uintptr_t>(p) - (uintptr_t)((int64_t)z0 * plane_elems * (int64_t)sizeof(double));
}

int Solver::slab_forward(const double* rhs) {
    if (!is_setup || !owned()) return -1;
    if (!rhs) return -2;
    int64_t ustr[3], ucstr;
    set_strides_user(ustr, ucstr);
    pass_idx = 0;
    slab_dim = 2;
    slab_lo = own[0];
    slab_hi = own[1];
    do_fft_forward(reinterpret_cast<const double*>(slab_base(rhs, own[0], ustr[2])), 1);
    slab_dim = -1;
    collect_timing();
    check_cuda(cudaGetLastError(), "slab forward");
    return 0;
}

int Solver::slab_fused(int type) {
    if (!is_setup || !owned()) return -1;
    if (int e = slab_check(type); e) return e;
    pass_idx = 0;
    slab_dim = 0;
    slab_lo = own[2];
    slab_hi = own[3];
    do_fused(type, 1);
    slab_dim = -1;
    collect_timing();
    check_cuda(cudaGetLastError(), "slab fused pass");
    return 0;
}

int Solver::slab_backward(double* field, int type) {
    if (!is_setup || !owned()) return -1;
    if (int e = slab_check(type); e) return e;
    if (!field) return -2;
    int64_t ustr[3], ucstr;
    set_strides_user(ustr, ucstr);
    pass_idx = 0;
    slab_dim = 2;
    slab_lo = own[0];
    slab_hi = own[1];
    do_backward(reinterpret_cast<double*>(slab_base(field, own[0], ustr[2])), type, 1);
    slab_dim = -1;
    collect_timing();
    if (!async) check_cuda(cudaStreamSynchronize(stream), "slab backward");
    else check_cuda(cudaGetLastError(), "slab backward");
    return 0;
}

// ---------------------------------------------------------------- advanced API
// flups_get_innerBuffer / flups_get_innerTopo_* / flups_do_copy / do_FFT /
// do_mult (Solver.cpp:518-530, 1281-1516).  The inner buffer is managed memory
// (host code may fill and read it, as the reference's samples do; kernels read
// it on the device) holding doubles in one of two layouts:
//   physical: the user layout of flups_topo_new (x fastest, lda slowest);
//   spectral: the full spectrum after every forward direction, complex,
//             x fastest with rows padded to 8 complex (128 bytes), lda slowest;
//             described by flups_get_innerTopo_spectral (axis 0, nf = 2).
// The transforms run on the solver's work arrays; the first and last passes
// read / write the doubles of the inner layouts.
void Solver::ensure_inner() {
    FLB_CHECK(is_setup, "flups_setup must be called before using the inner buffer");
    const ArrState& S = st[ndim];
    inner_pitch = ((int64_t)S.n[0] + 7) / 8 * 8;
    const size_t spec = (size_t)inner_pitch * S.n[1] * S.n[2] * 2 * lda;
    const size_t need = std::max(spec, topo_phys->memsize());
    if (!inner || inner_elems < need) {
        if (inner) cudaFree(inner);
        inner = nullptr;
        check_cuda(cudaMallocManaged(&inner, need * sizeof(double)), "inner buffer");
        check_cuda(cudaMemset(inner, 0, need * sizeof(double)), "inner buffer");
        inner_elems = need;
    }
    if (!topo_inner_phys) topo_inner_phys = new Topology(*topo_phys);
    if (!topo_spec) {
        topo_spec = new Topology(*topo_phys);
        topo_spec->axis = 0;
        topo_spec->nf = 2;
        for (int d = 0; d < 3; ++d) {
            topo_spec->nglob[d] = S.n[d];
            topo_spec->nloc[d] = S.n[d];
            topo_spec->nmem[d] = S.n[d];
        }
        topo_spec->nmem[0] = (int)inner_pitch;
    }
}

void Solver::inner_spec_strides(int64_t str[3], int64_t& cstr) const {
    const ArrState& S = st[ndim];
    str[0] = 1;
    str[1] = inner_pitch;
    str[2] = inner_pitch * S.n[1];
    cstr = inner_pitch * S.n[1] * S.n[2];
}

void Solver::adv_copy(const Topology* topo, double* data, int sign) {
    cs_follows = false;
    FLB_CHECK(data != nullptr, "data is NULL");
    FLB_CHECK(topo != nullptr && topo->lda == lda, "the solver lda = %d must match the topology one", lda);
    FLB_CHECK(topo->memsize() == topo_phys->memsize(), "the topology must be the solver's physical topology");
    ensure_inner();
    const size_t bytes = topo->memsize() * sizeof(double);
    if (sign == FLUPS_FORWARD)
        check_cuda(cudaMemcpyAsync(inner, data, bytes, cudaMemcpyDefault, stream), "copy to the inner buffer");
    else
        check_cuda(cudaMemcpyAsync(data, inner, bytes, cudaMemcpyDefault, stream), "copy from the inner buffer");
    check_cuda(cudaStreamSynchronize(stream), "copy");
}

void Solver::adv_fft(double* data, int sign) {
    cs_follows = false;
    FLB_CHECK(data != nullptr, "data is NULL");
    FLB_CHECK(!owned(), "this solver holds one rank's share of the planes: use the flups_b200_slab_* steps");
    FLB_CHECK(sign == FLUPS_FORWARD || sign == FLUPS_BACKWARD || sign == FLUPS_BACKWARD_DIFF, "unknown sign %d", sign);
    FLB_CHECK(sign != FLUPS_BACKWARD_DIFF || have_diff, "FLUPS_BACKWARD_DIFF needs a solver set up with a derivative order");
    ensure_inner();
    ensure_buffers(1);
    const bool f64 = (precision == 64);
    const int es = f64 ? 8 : 4;
    pass_idx = 0;
    if (sign == FLUPS_FORWARD) {
        for (int ip = 0; ip < ndim; ++ip) {
            const DirPlan& p = fwd[ip];
            PassArgs A = base_pass(p.dim, st[ip], lda, lda);
            A.st[0] = stage_forward(p, ip, f64);
            if (ip == 0) {
                set_strides_user(A.in_str, A.in_cstr);
                A.in = data;
            } else {
                set_strides_internal(A.in_str, A.in_cstr, st[ip]);
                A.in = buf[(ip - 1) % 2];
            }
            if (ip == ndim - 1) {
                inner_spec_strides(A.out_str, A.out_cstr);
                A.out = data;
            } else {
                set_strides_internal(A.out_str, A.out_cstr, st[ip + 1]);
                A.out = buf[ip % 2];
            }
            fit_lines(A, es);
            run_pass(A, f64, ip == 0 ? true : f64, ip == ndim - 1 ? true : f64, "adv_fwd");
        }
    } else {
        for (int ip = ndim - 1; ip >= 0; --ip) {
            const DirPlan& p = (sign == FLUPS_BACKWARD_DIFF) ? dif[ip] : bwd[ip];
            PassArgs A = base_pass(fwd[ip].dim, st[ip + 1], lda, lda);
            A.st[0] = stage_backward(p, fwd[ip], ip, f64);
            if (ip == ndim - 1) {
                inner_spec_strides(A.in_str, A.in_cstr);
                A.in = data;
            } else {
                set_strides_internal(A.in_str, A.in_cstr, st[ip + 1]);
                A.in = buf[ip % 2];
            }
            if (ip == 0) {
                set_strides_user(A.out_str, A.out_cstr);
                A.out = data;
            } else {
                set_strides_internal(A.out_str, A.out_cstr, st[ip]);
                A.out = buf[(ip - 1) % 2];
            }
            fit_lines(A, es);
            run_pass(A, f64, ip == ndim - 1 ? true : f64, ip == 0 ? true : f64, "adv_bwd");
        }
    }
    check_cuda(cudaStreamSynchronize(stream), "flups_do_FFT");
}

void Solver::adv_mult(double* data, int type) {
    cs_follows = false;
    FLB_CHECK(data != nullptr, "data is NULL");
    FLB_CHECK(type == STD || (type == ROT && lda == 3 && odiff != NOD), "ROT needs lda = 3 and a derivative order");
    ensure_inner();
    RotArgs R;
    memset(&R, 0, sizeof(R));
    R.data = data;
    for (int d = 0; d < 3; ++d) R.n[d] = st[ndim].n[d];
    inner_spec_strides(R.str, R.cstr);
    R.nbatch = 1;
    R.ncomp = lda;
    R.mult = mult_spec(type);
    check_cuda(launch_spec_mult(R, 1, precision == 64 ? 1 : 0, stream), "flups_do_mult");
    check_cuda(cudaStreamSynchronize(stream), "flups_do_mult");
}

// ---------------------------------------------------------------- autotuning
std::string Solver::pass_key(const PassArgs& A, bool f64) const {
    char b[160];
    snprintf(b, sizeof(b), "%d/%d/%d/%d/%d/%d/%d/%d/%d", f64 ? 1 : 0, A.axis, A.fused, A.st[0].M, A.n_src,
             A.st[A.fused ? 1 : 0].n_store, A.n_a, A.n_b, A.ncomp);
    return b;
}

// Time both CTA tiles of every column pass of a (type, nbatch) solve and keep
// the faster.  The passes run on the solver's work arrays, whose contents are
// dead between solves (the real passes overwrite them), so tuning needs no
// extra memory; it synchronises the stream and runs once per signature.
void Solver::autotune_passes(int type, int nbatch) {
    const int64_t sk = (int64_t)nbatch * 4 + type;
    if (tuned_solves.count(sk)) return;
    tuned_solves[sk] = true;
    const bool f64 = (precision == 64);
    dry = true;
    dry_passes.clear();
    dry_flags.clear();
    dry_names.clear();
    dry_fast.clear();
    do_fft_forward(nullptr, nbatch);
    do_fft_backward_fused(nullptr, type, nbatch);
    dry = false;
    std::vector<PassArgs> passes = dry_passes;
    std::vector<int> kinds = dry_fast;
    dry_passes.clear();
    dry_flags.clear();
    dry_names.clear();
    dry_fast.clear();
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "event");
    check_cuda(cudaEventCreate(&e1), "event");
    for (size_t i = 0; i < passes.size(); ++i) {
        if (kinds[i] != 1) continue;
        const PassArgs& A = passes[i];
        const std::string key = pass_key(A, f64);
        if (tuned_tile.count(key)) continue;
        ColArgs c;
        RowArgs r;
        int mode = 0;
        fast_args(A, 1, f64, f64, c, r, mode);
        const int L = A.st[0].M;
        c.tws = stage_table(L, f64, fast_radix1_mode(L, f64 ? 1 : 0, mode));
        float best = 1e30f;
        int best_tile = COL_TILE_DEFAULT;
        for (int tile : {COL_TILE_256, COL_TILE_128}) {
            c.tile = tile;
            check_cuda(launch_fast_col(f64, mode, L, c, A.ncomp, stream), "autotune launch");
            check_cuda(cudaEventRecord(e0, stream), "event");
            for (int k = 0; k < 3; ++k) check_cuda(launch_fast_col(f64, mode, L, c, A.ncomp, stream), "autotune launch");
            check_cuda(cudaEventRecord(e1, stream), "event");
            check_cuda(cudaEventSynchronize(e1), "autotune");
            float ms = 0.f;
            check_cuda(cudaEventElapsedTime(&ms, e0, e1), "event");
            if (ms < best) {
                best = ms;
                best_tile = tile;
            }
        }
        tuned_tile[key] = best_tile;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// ---------------------------------------------------------------- CUDA graphs
// A solve of device arrays is a fixed sequence of launches on the solver's
// stream, so it can be captured once and replayed: the first call for a given
// (field, rhs, nbatch, type) runs a plain solve (which allocates and tunes what
// it needs), then captures a second one; later calls only launch the graph.
int Solver::solve_graph(double* field, double* rhs, int type, int nbatch) {
    if (!is_setup || !field || !rhs || nbatch < 1 || owned()) return -1;
    if (!is_device_ptr(field) || !is_device_ptr(rhs)) return -2;
    cs_follows = false;
    GraphKey k{field, rhs, nbatch, type};
    auto it = graphs.find(k);
    if (it == graphs.end()) {
        const bool keep_async = async;
        async = true;
        solve(field, rhs, type, nbatch);  // allocations, tuning, kernel attributes
        // capture on a private stream (the legacy default stream cannot be captured)
        if (!capture_stream) check_cuda(cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking), "capture stream");
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        cudaStream_t user_stream = stream;
        stream = capture_stream;
        capturing = true;
        cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            solve(field, rhs, type, nbatch);
            e = cudaStreamEndCapture(stream, &g);
        }
        capturing = false;
        stream = user_stream;
        async = keep_async;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            last_error = (int)e;
            cudaGetLastError();
            return -4;
        }
        it = graphs.emplace(k, ge).first;
    }
    const cudaError_t e = cudaGraphLaunch(it->second, stream);
    if (e != cudaSuccess) {
        last_error = (int)e;
        return -4;
    }
    if (!async) check_cuda(cudaStreamSynchronize(stream), "graph solve");
    return 0;
}

// ---------------------------------------------------------------- host-only description
static void json_plan(std::string& o, const DirPlan& p) {
    char b[1024];
    snprintf(b, sizeof(b),
             "{\"dim\":%d,\"type\":%d,\"n_out\":%d,\"fieldstart\":%d,\"koffset\":%.17g,\"kfact\":%.17g,\"symstart\":%.17g,"
             "\"normfact\":%.17g,\"volfact\":%.17g,\"isr2c\":%d,\"is_spectral\":%d,\"comp\":[",
             p.dim, p.type, p.n_out, p.fieldstart, p.koffset, p.kfact, p.symstart, p.normfact, p.volfact, p.isr2c ? 1 : 0,
             p.is_spectral ? 1 : 0);
    o += b;
    for (int c = 0; c < p.lda; ++c) {
        snprintf(b, sizeof(b), "%s{\"n_in\":%d,\"fi\":%d,\"fo\":%d,\"postpro\":%d,\"imult\":%d,\"kind\":%d}", c ? "," : "",
                 p.n_in[c], p.fstart_in[c], p.fstart_out[c], p.postpro[c], p.imult[c] ? 1 : 0, p.kind[c]);
        o += b;
    }
    o += "]}";
}

std::string Solver::plan_json(int type, int nbatch) {
    std::string o = "{";
    char b[512];
    snprintf(b, sizeof(b), "\"ndim\":%d,\"normfact\":%.17g,\"volfact\":%.17g,\"plans\":{", ndim, normfact, volfact);
    o += b;
    const char* names[4] = {"fwd", "bwd", "grn", "dif"};
    DirPlan* sets[4] = {fwd, bwd, grn, dif};
    for (int k = 0; k < (have_diff ? 4 : 3); ++k) {
        o += (k ? ",\"" : "\"");
        o += names[k];
        o += "\":[";
        for (int ip = 0; ip < 3; ++ip) {
            if (ip) o += ",";
            json_plan(o, sets[k][ip]);
        }
        o += "]";
    }
    o += "},\"states\":[";
    for (int k = 0; k <= ndim; ++k) {
        snprintf(b, sizeof(b), "%s[%d,%d,%d,%d]", k ? "," : "", st[k].n[0], st[k].n[1], st[k].n[2], st[k].cplx ? 1 : 0);
        o += b;
    }
    o += "],\"passes\":[";
    dry = true;
    dry_passes.clear();
    dry_flags.clear();
    dry_names.clear();
    dry_fast.clear();
    compute_green();
    plan_xlast();
    // the passes of a solve of device arrays (the x-last order where it applies)
    const bool xl = xlast_ok(type);
    if (xl) swap_order();
    do_fft_forward(nullptr, nbatch);
    do_fft_backward_fused(nullptr, type, nbatch);
    if (xl) swap_order();
    dry = false;
    for (size_t i = 0; i < dry_passes.size(); ++i) {
        const PassArgs& A = dry_passes[i];
        const int es = (dry_flags[i] & 1) ? 8 : 4;
        snprintf(b, sizeof(b),
                 "%s{\"name\":\"%s\",\"axis\":%d,\"n_src\":%d,\"n_a\":%d,\"n_b\":%d,\"ncomp\":%d,\"lda\":%d,\"lines_per_cta\":%d,"
                 "\"fused\":%d,\"comps_together\":%d,\"flags\":%d,\"fast\":%d,\"smem\":%zu,\"st\":[",
                 i ? "," : "", dry_names[i].c_str(), A.axis, A.n_src, A.n_a, A.n_b, A.ncomp, A.lda, A.lines_per_cta, A.fused,
                 A.comps_together, dry_flags[i], dry_fast[i], line_pass_smem(A, es));
        o += b;
        for (int s2 = 0; s2 <= A.fused; ++s2) {
            const LineStage& S = A.st[s2];
            snprintf(b, sizeof(b),
                     "%s{\"M\":%d,\"nrad\":%d,\"n_b\":%d,\"fieldstart\":%d,\"n_o\":%d,\"in_cplx\":%d,\"out_cplx\":%d,"
                     "\"store_off\":%d,\"n_store\":%d,\"spec\":[",
                     s2 ? "," : "", S.M, S.nrad, S.n_b, S.fieldstart, S.n_o, S.in_cplx, S.out_cplx, S.store_off, S.n_store);
            o += b;
            for (int c = 0; c < lda; ++c) {
                const LineSpec& sp = S.spec[c];
                snprintf(b, sizeof(b), "%s{\"kind\":%d,\"sign\":%d,\"n_in\":%d,\"fi\":%d,\"fo\":%d,\"postpro\":%d,\"nfftw\":%d}",
                         c ? "," : "", sp.kind, sp.sign, sp.n_in, sp.fi, sp.fo, sp.postpro, sp.nfftw);
                o += b;
            }
            o += "]}";
        }
        o += "]}";
    }
    o += "],\"xlast\":";
    o += xl ? "1" : "0";
    o += "}";
    return o;
}
