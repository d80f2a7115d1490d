// extern "C" entry points of libflups_b200.so: the reference's C API
// (src/flups.h, implemented there by src/flups.cpp:17-343) on top of the
// B200 solver, plus the additive entry points of include/flups_b200.h.
#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <string>

#include "host.hpp"

extern "C" {

// ---------------------------------------------------------------- memory
void* flups_malloc(size_t size) {
    // flups.cpp:19-21: aligned, zeroed host memory
    void* p = nullptr;
    if (posix_memalign(&p, 64, size ? size : 64) != 0) return nullptr;
    memset(p, 0, size);
    return p;
}

void flups_free(void* data) { free(data); }

void flups_info(int argc, char** argv) {
    // flups.cpp:257-341: bookkeeping file next to the executable name
    std::string fn(argc > 0 && argv && argv[0] ? argv[0] : "flups");
    std::string clean;
    for (char c : fn)
        if (c != '.' && c != '/') clean += c;
    clean += ".flups.info";
    FILE* f = fopen(clean.c_str(), "w+");
    if (!f) return;
    fprintf(f, "FLUPS (B200 library)\n- comm_world size: 1\n- defines:\n\tFLUPS_ALIGNMENT = %d\n", FLUPS_ALIGNMENT);
    int dev = -1;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (dev >= 0 && cudaGetDeviceProperties(&prop, dev) == cudaSuccess) fprintf(f, "\tdevice = %s (sm_%d%d)\n", prop.name, prop.major, prop.minor);
    fprintf(f, "- argument list:\n");
    for (int i = 1; i < argc; ++i) fprintf(f, "\t%s\n", argv[i]);
    fclose(f);
}

// ---------------------------------------------------------------- topologies
void Topology::cmpt_sizes() {
    // Topology.cpp:81-98: pad the axis so that every pencil starts aligned
    for (int id = 0; id < 3; ++id) {
        nloc[id] = nglob[id] / nproc[id] + ((nglob[id] % nproc[id]) > 0 ? 1 : 0);
        nmem[id] = nloc[id];
        if (id == axis) {
            const int modulo = (int)((nloc[id] * nf * sizeof(double)) % alignment);
            const int delta = (int)((alignment - modulo) / sizeof(double));
            nmem[id] += (modulo == 0) ? 0 : delta / nf;
        }
    }
}

Topology* flups_topo_new(const int axis, const int lda, const int nglob[3], const int nproc[3], const bool isComplex,
                         const int axproc[3], const int alignment, MPI_Comm comm) {
    FLB_CHECK(axis >= 0 && axis < 3, "axis must be 0, 1 or 2");
    FLB_CHECK(nproc[0] * nproc[1] * nproc[2] == 1, "the total number of procs (=%d) have to be = to the comm size (=1)",
              nproc[0] * nproc[1] * nproc[2]);
    FLB_CHECK(alignment > 0 && alignment % (int)sizeof(double) == 0, "alignment must be a multiple of 8 bytes");
    Topology* t = new Topology();
    t->axis = axis;
    t->lda = lda;
    t->nf = isComplex ? 2 : 1;
    t->alignment = alignment;
    t->comm = comm;
    for (int d = 0; d < 3; ++d) {
        t->nglob[d] = nglob[d];
        t->nproc[d] = nproc[d];
        t->axproc[d] = axproc ? axproc[d] : d;
    }
    t->cmpt_sizes();
    return t;
}

Topology* flups_init_topology(const int axis, const int lda, const int nglob[3], const int nproc[3], const bool isComplex,
                              const int axproc[3], const int alignment, MPI_Comm comm) {
    return flups_topo_new(axis, lda, nglob, nproc, isComplex, axproc, alignment, comm);
}

void flups_topo_free(const Topology* t) { delete t; }
bool flups_topo_get_isComplex(const Topology* t) { return t->nf == 2; }
int flups_topo_get_lda(const Topology* t) { return t->lda; }
int flups_topo_get_axis(const Topology* t) { return t->axis; }
int flups_topo_get_nglob(const Topology* t, const int dim) { return t->nglob[dim]; }
int flups_topo_get_nloc(const Topology* t, const int dim) { return t->nloc[dim]; }
int flups_topo_get_nmem(const Topology* t, const int dim) { return t->nmem[dim]; }
int flups_topo_get_nproc(const Topology* t, const int dim) { return t->nproc[dim]; }
void flups_topo_get_istartGlob(const Topology* t, int istart[3]) {
    (void)t;
    istart[0] = istart[1] = istart[2] = 0;
}
size_t flups_topo_get_locsize(const Topology* t) { return t->locsize(); }
size_t flups_topo_get_memsize(const Topology* t) { return t->memsize(); }
int flups_topo_cmpt_rank_fromid(const Topology* t, const int global_id, const int id) {
    (void)t; (void)global_id; (void)id;
    return 0;
}
int flups_topo_cmpt_start_id_from_rank(const Topology* t, const int rank_id, const int id) {
    // Topology.hpp:113-125 (balanced split) with the topology's nproc
    const int b = t->nglob[id] / t->nproc[id];
    const int res = t->nglob[id] % t->nproc[id];
    const int s = (res > 0) ? (t->nproc[id] / res) : 0x7fffffff;
    const int q = rank_id / s;
    return rank_id * b + (q < res ? q : res);
}
MPI_Comm flups_topo_get_comm(Topology* t) { return t->comm; }
void flups_topo_ranksplit(const Topology* t, const int rank, int rankd[3]) {
    (void)t; (void)rank;
    rankd[0] = rankd[1] = rankd[2] = 0;
}
int flups_topo_rankindex(const Topology* topo, const int rankd[3]) {
    (void)topo;
    return rankd[0] + rankd[1] + rankd[2];
}

// ---------------------------------------------------------------- solver
Solver* flups_init(Topology* t, FLUPS_BoundaryType* bc[3][2], const double h[3], const double L[3], FLUPS_DiffType orderDiff,
                   const FLUPS_CenterType center_type[3]) {
    const int c[3] = {center_type[0], center_type[1], center_type[2]};
    return new Solver(t, bc, h, L, orderDiff, c, nullptr);
}

Solver* flups_init_timed(Topology* t, FLUPS_BoundaryType* bc[3][2], const double h[3], const double L[3], const FLUPS_DiffType orderDiff,
                         const FLUPS_CenterType center_type[3], Profiler* prof) {
    const int c[3] = {center_type[0], center_type[1], center_type[2]};
    return new Solver(t, bc, h, L, orderDiff, c, prof);
}

void flups_cleanup_solver(Solver* s) { delete s; }
void flups_cleanup_backend(void) {}
void flups_cleanup_all(Solver* s) {
    delete s;
    flups_cleanup_backend();
}
void flups_cleanup(Solver* s) { flups_cleanup_all(s); }

void flups_set_greenType(Solver* s, const FLUPS_GreenType type) {
    FLB_CHECK(!s->is_setup, "the Green's function type must be set before flups_setup");
    s->green_type = type;
}

void flups_set_stream(Solver* s, void* stream) {
    s->stream = (cudaStream_t)stream;
    s->cs_follows = false;
}

void flups_setup(Solver* s, const bool changeComm) {
    (void)changeComm;
    auto t0 = std::chrono::steady_clock::now();
    s->setup();
    if (s->prof) {
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        s->prof->acc_ms["setup"] += ms;
        s->prof->count["setup"] += 1;
    }
}

static void timed_solve(Solver* s, double* field, double* rhs, int type, int nbatch) {
    if (!s->prof) {
        s->solve(field, rhs, type, nbatch);
        return;
    }
    auto t0 = std::chrono::steady_clock::now();
    s->solve(field, rhs, type, nbatch);
    cudaStreamSynchronize(s->stream);
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    s->prof->acc_ms["solve"] += ms;
    s->prof->count["solve"] += 1;
}

void flups_solve(Solver* s, double* field, double* rhs, const FLUPS_SolverType type) { timed_solve(s, field, rhs, type, 1); }
void flups_synchronize(Solver* s) { s->check_cuda(cudaStreamSynchronize(s->stream), "synchronize"); }
void flups_solve_rot(Solver* s, double* field, double* rhs) { timed_solve(s, field, rhs, ROT, 1); }
void flups_solve_batch(Solver* s, double* field, double* rhs, int nbatch, int type) { timed_solve(s, field, rhs, type, nbatch); }

// ---------------------------------------------------------------- advanced
size_t flups_get_allocSize(Solver* s) { return s->alloc_size(); }
void flups_get_spectralInfo(Solver* s, double kfact[3], double koffset[3], double symstart[3]) {
    s->spectral_info(kfact, koffset, symstart);
}
void flups_set_alpha(Solver* s, const double alpha) {
    FLB_CHECK(!s->is_setup, "alpha must be set before flups_setup");
    s->alpha = alpha;
}
double* flups_get_innerBuffer(Solver* s) {
    s->ensure_inner();
    return s->inner;
}
Topology* flups_get_innerTopo_physical(Solver* s) {
    s->ensure_inner();
    return s->topo_inner_phys;
}
Topology* flups_get_innerTopo_spectral(Solver* s) {
    s->ensure_inner();
    return s->topo_spec;
}
// the inner physical layout is the user layout: there is no first topology
// switch to skip (kept as a no-op flag for callers of the reference API)
void flups_skip_firstSwitchtopo(Solver* s) { s->skip_st0 = true; }
void flups_do_copy(Solver* s, const Topology* topo, double* data, const int sign) { s->adv_copy(topo, data, sign); }
void flups_do_FFT(Solver* s, double* data, const int sign) { s->adv_fft(data, sign); }
void flups_do_mult(Solver* s, double* data, const FLUPS_SolverType type) { s->adv_mult(data, type); }

void flups_pencilDirs(const FLUPS_BoundaryType* bc[3][2], int dirs[3]) {
    // flups.cpp:200-211: directions sorted (stably) by plan type
    int t[3];
    for (int d = 0; d < 3; ++d) t[d] = bc[d][0][0] + bc[d][1][0];
    int o[3] = {0, 1, 2};
    for (int i = 1; i < 3; ++i)
        for (int j = i; j > 0 && t[o[j]] < t[o[j - 1]]; --j) std::swap(o[j], o[j - 1]);
    for (int i = 0; i < 3; ++i) dirs[i] = o[i];
}

void flups_switchtopo_info(Solver* s) {
    printf("flups_b200: no pencil switches; %d line passes per solve (directions", 2 * s->ndim - 1);
    for (int ip = 0; ip < s->ndim; ++ip) printf(" %d", s->fwd[ip].dim);
    printf(")\n");
}

// ---------------------------------------------------------------- additive
void flups_set_precision(Solver* s, int bits) {
    FLB_CHECK(!s->is_setup, "precision must be set before flups_setup");
    FLB_CHECK(bits == 32 || bits == 64, "precision must be 32 or 64 bits");
    s->precision = bits;
}
int flups_get_precision(Solver* s) { return s->precision; }
void flups_set_async(Solver* s, int async) { s->async = async != 0; }
// switches that change the passes drop the captured solves
void flups_b200_set_fast_kernels(Solver* s, int on) {
    s->use_fast = on != 0;
    s->drop_graphs();
}
void flups_b200_set_autotune(Solver* s, int on) {
    s->autotune = on != 0;
    s->drop_graphs();
}
void flups_b200_set_overlap(Solver* s, int on) {
    s->overlap = on != 0;
    s->drop_graphs();
}
void flups_b200_set_prefetch(Solver* s, int on) {
    s->prefetch = on != 0;
    s->drop_graphs();
}
void flups_b200_set_xlast(Solver* s, int on) {
    s->xlast_on = on != 0;
    s->drop_graphs();
}
void flups_b200_set_col_tile(Solver* s, int tile) {
    s->force_tile = (tile == 1 || tile == 2) ? tile : 0;
    s->drop_graphs();
}
int flups_solve_graph(Solver* s, double* field, double* rhs, int nbatch, int type) {
    if (!s) return -1;
    return s->solve_graph(field, rhs, type, nbatch);
}
int flups_get_last_error(Solver* s) { return s->last_error; }

int flups_b200_slab_info(Solver* s, int64_t info[7]) {
    if (!s || !info) return -1;
    const int e = s->slab_check(STD);
    const ArrState& sp = s->st[s->ndim - 1];
    info[0] = sp.n[0];
    info[1] = sp.n[1];
    info[2] = sp.n[2];
    info[3] = s->row_pitch(sp);
    info[4] = s->st[0].n[2];
    info[5] = s->xpitch;
    info[6] = (s->precision == 64) ? 8 : 4;
    return e;
}
int flups_b200_slab_own(Solver* s, int z0, int z1, int x0, int x1) { return s ? s->slab_own(z0, z1, x0, x1) : -1; }
void* flups_b200_slab_planes(Solver* s) { return (s && s->owned() && s->is_setup) ? s->buf[(s->ndim - 2) % 2] : nullptr; }
void* flups_b200_slab_columns(Solver* s) { return (s && s->owned() && s->is_setup) ? s->xbuf : nullptr; }
int flups_b200_slab_forward(Solver* s, const double* rhs) { return s ? s->slab_forward(rhs) : -1; }
int flups_b200_slab_fused(Solver* s, int type) { return s ? s->slab_fused(type) : -1; }
int flups_b200_slab_backward(Solver* s, double* field, int type) { return s ? s->slab_backward(field, type) : -1; }
int flups_b200_slab_peers(Solver* s, int n, void* const* cols, const int* xs, const int64_t* pitch) {
    return s ? s->slab_peers(n, cols, xs, pitch) : -1;
}
int flups_b200_ipc_handle(const void* dev_ptr, void* handle) {
    if (!dev_ptr || !handle) return -2;
    cudaIpcMemHandle_t h;
    if (cudaIpcGetMemHandle(&h, const_cast<void*>(dev_ptr)) != cudaSuccess) {
        cudaGetLastError();
        return -4;
    }
    memcpy(handle, &h, sizeof(h));
    return 0;
}
int flups_b200_ipc_open(const void* handle, void** dev_ptr) {
    if (!handle || !dev_ptr) return -2;
    cudaIpcMemHandle_t h;
    memcpy(&h, handle, sizeof(h));
    if (cudaIpcOpenMemHandle(dev_ptr, h, cudaIpcMemLazyEnablePeerAccess) != cudaSuccess) {
        cudaGetLastError();
        return -4;
    }
    return 0;
}
int flups_b200_ipc_close(void* dev_ptr) { return cudaIpcCloseMemHandle(dev_ptr) == cudaSuccess ? 0 : -4; }
size_t flups_get_device_bytes(Solver* s, int nbatch) { return s->device_bytes(nbatch); }

int flups_b200_plan_json(Solver* s, int type, int nbatch, char* out, int len) {
    const std::string j = s->plan_json(type, nbatch);
    if (out && len > 0) {
        strncpy(out, j.c_str(), len - 1);
        out[len - 1] = 0;
    }
    return (int)j.size() + 1;
}

void flups_set_pass_timing(Solver* s, int on) {
    s->timing = on != 0;
    s->pass_ms.assign(s->pass_ms.size(), 0.0);
    s->pass_calls.assign(s->pass_calls.size(), 0);
}

int flups_get_pass_stats(Solver* s, int maxn, double* ms_total, double* bytes, long* calls, char* names, int name_len) {
    const int n = (int)s->pass_ms.size();
    for (int k = 0; k < n && k < maxn; ++k) {
        if (ms_total) ms_total[k] = s->pass_ms[k];
        if (bytes) bytes[k] = s->pass_bytes[k];
        if (calls) calls[k] = s->pass_calls[k];
        if (names && name_len > 0) {
            strncpy(names + (size_t)k * name_len, s->pass_names[k].c_str(), name_len - 1);
            names[(size_t)k * name_len + name_len - 1] = 0;
        }
    }
    return n;
}

// ---------------------------------------------------------------- profiler
Profiler* flups_profiler_new(void) {
    Profiler* p = new Profiler();
    p->name = "default";
    return p;
}
Profiler* flups_profiler_new_n(const char name[]) {
    Profiler* p = new Profiler();
    p->name = name ? name : "default";
    return p;
}
void flups_profiler_free(Profiler* p) { delete p; }
void flups_profiler_disp(Profiler* p) {
    if (!p) return;
    printf("===== profiler %s =====\n", p->name.c_str());
    for (auto& kv : p->acc_ms) {
        const long n = p->count[kv.first];
        printf("  %-10s calls %6ld  total %10.3f ms  mean %10.3f ms\n", kv.first.c_str(), n, kv.second, n ? kv.second / n : 0.0);
    }
}

// ---------------------------------------------------------------- output
void flups_hdf5_dump(const Topology* topo, const char filename[], const double* data) {
    // The reference writes HDF5 + XDMF (src/hdf5_io.cpp:11-246); HDF5 is not
    // available here, so the same field goes to ./data/<name>.bin (raw
    // doubles, memory layout of the topology) with an XDMF description.
    mkdir("./data", 0770);
    const std::string base = std::string("./data/") + filename;
    FILE* f = fopen((base + ".bin").c_str(), "wb");
    if (!f) return;
    fwrite(data, sizeof(double), topo->memsize(), f);
    fclose(f);
    FILE* x = fopen((base + ".xmf").c_str(), "w");
    if (!x) return;
    fprintf(x, "<?xml version=\"1.0\" ?>\n<Xdmf Version=\"2.0\">\n <Domain>\n  <Grid Name=\"%s\">\n", filename);
    fprintf(x, "   <Topology TopologyType=\"3DCoRectMesh\" Dimensions=\"%d %d %d\"/>\n", topo->nmem[2], topo->nmem[1], topo->nmem[0]);
    fprintf(x, "   <Attribute Name=\"data\"><DataItem Dimensions=\"%d %d %d %d\" NumberType=\"Float\" Precision=\"8\" Format=\"Binary\">%s.bin</DataItem></Attribute>\n",
            topo->lda, topo->nmem[2], topo->nmem[1], topo->nmem[0] * topo->nf, filename);
    fprintf(x, "  </Grid>\n </Domain>\n</Xdmf>\n");
    fclose(x);
}

void flups_print_data(const Topology* topo, double* data) {
    const int ax0 = topo->axis, ax1 = (ax0 + 1) % 3, ax2 = (ax0 + 2) % 3;
    for (int lia = 0; lia < topo->lda; ++lia)
        for (int i2 = 0; i2 < topo->nloc[ax2]; ++i2)
            for (int i1 = 0; i1 < topo->nloc[ax1]; ++i1) {
                for (int i0 = 0; i0 < topo->nloc[ax0]; ++i0) {
                    const size_t id = flups_locID(ax0, i0, i1, i2, lia, ax0, topo->nmem, topo->nf);
                    if (topo->nf == 2) printf("(%+.6e,%+.6e) ", data[id], data[id + 1]);
                    else printf("%+.6e ", data[id]);
                }
                printf("\n");
            }
}

}  // extern "C"
