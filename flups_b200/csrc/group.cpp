// Solves of several solvers -- unevenly sized grids, different boundary
// conditions, kernels, precisions or solver types -- replayed as ONE CUDA
// graph (flups_b200_solve_group).  The first call for a given set of
// (solver, field, rhs, type) runs each solve once (allocations, tuning,
// kernel attributes), then captures all of them into one graph whose member
// solves are independent branches (forked from one capture stream, each on a
// stream of its own, joined at the end), so the small grids' passes run side
// by side on the GPU; later calls launch that graph.  A member whose work
// arrays were reallocated or whose switches changed since (Solver::gen) gets
// the group recaptured; a destroyed member drops every group it was in.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <vector>

#include "host.hpp"

namespace {

struct GroupGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> gens;
};

std::mutex g_mu;
std::map<std::vector<uintptr_t>, GroupGraph> g_groups;

bool is_device(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

namespace flb {

void group_forget(const Solver* s) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto it = g_groups.begin(); it != g_groups.end();) {
        const std::vector<uintptr_t>& k = it->first;
        const size_t n = k.empty() ? 0 : k[0];
        bool holds = false;
        for (size_t i = 0; i < n; ++i) holds = holds || k[1 + i] == reinterpret_cast<uintptr_t>(s);
        if (holds) {
            cudaGraphExecDestroy(it->second.exec);
            it = g_groups.erase(it);
        } else {
            ++it;
        }
    }
}

}  // namespace flb

// Captures the members' solves as branches of one graph; 0 or a CUDA error.
static cudaError_t capture_group(Solver* const* ss, int n, double* const* fields, double* const* rhss, const int* types,
                                 cudaGraphExec_t* exec) {
    cudaStream_t origin = nullptr;
    std::vector<cudaStream_t> branch(n, nullptr);
    std::vector<cudaEvent_t> join(n, nullptr);
    cudaEvent_t fork = nullptr;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        e = cudaStreamCreateWithFlags(&branch[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t ce = cudaEventRecord(fork, origin);
        for (int i = 0; i < n && ce == cudaSuccess; ++i) {
            Solver* s = ss[i];
            ce = cudaStreamWaitEvent(branch[i], fork, 0);
            if (ce != cudaSuccess) break;
            const cudaStream_t keep_stream = s->stream;
            const bool keep_async = s->async, keep_timing = s->timing;
            s->stream = branch[i];
            s->async = true;
            s->timing = false;  // no event waits inside a capture
            s->capturing = true;
            s->solve(fields[i], rhss[i], types[i], 1);
            s->capturing = false;
            s->timing = keep_timing;
            s->async = keep_async;
            s->stream = keep_stream;
            ce = cudaEventRecord(join[i], branch[i]);
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(origin, join[i], 0);
        }
        e = cudaStreamEndCapture(origin, &g);
        if (e == cudaSuccess) e = ce;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    if (g) cudaGraphDestroy(g);
    for (int i = 0; i < n; ++i) {
        if (join[i]) cudaEventDestroy(join[i]);
        if (branch[i]) cudaStreamDestroy(branch[i]);
    }
    if (fork) cudaEventDestroy(fork);
    if (origin) cudaStreamDestroy(origin);
    return e;
}

extern "C" int flups_b200_solve_group(Solver* const* ss, int n, double* const* fields, double* const* rhss, const int* types,
                                      void* stream) {
    if (!ss || !fields || !rhss || !types || n < 1 || n > 4096) return -1;
    for (int i = 0; i < n; ++i) {
        if (!ss[i] || !ss[i]->is_setup || ss[i]->owned() || !fields[i] || !rhss[i]) return -1;
        if (types[i] != STD && types[i] != ROT) return -1;
        // the branches run side by side: no solver twice (its work arrays are
        // one set), no output twice
        for (int j = 0; j < i; ++j)
            if (ss[j] == ss[i] || fields[j] == fields[i]) return -2;
        if (!is_device(fields[i]) || !is_device(rhss[i])) return -2;
    }
    std::vector<uintptr_t> key;
    key.reserve(1 + 4 * (size_t)n);
    key.push_back((uintptr_t)n);
    for (int i = 0; i < n; ++i) key.push_back(reinterpret_cast<uintptr_t>(ss[i]));
    for (int i = 0; i < n; ++i) key.push_back(reinterpret_cast<uintptr_t>(fields[i]));
    for (int i = 0; i < n; ++i) key.push_back(reinterpret_cast<uintptr_t>(rhss[i]));
    for (int i = 0; i < n; ++i) key.push_back((uintptr_t)types[i]);
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_groups.find(key);
    bool stale = it == g_groups.end();
    for (int i = 0; !stale && i < n; ++i) stale = it->second.gens[i] != ss[i]->gen;
    if (stale) {
        // plain solves first: whatever a solve allocates or tunes happens
        // outside the capture (they run on the members' streams, after the
        // work the caller queued on `stream`)
        if (const cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream)); e != cudaSuccess) {
            for (int i = 0; i < n; ++i) ss[i]->last_error = (int)e;
            return -4;
        }
        for (int i = 0; i < n; ++i) {
            const bool keep_async = ss[i]->async;
            ss[i]->async = false;
            ss[i]->solve(fields[i], rhss[i], types[i], 1);
            ss[i]->async = keep_async;
        }
        if (it != g_groups.end()) {
            cudaGraphExecDestroy(it->second.exec);
            g_groups.erase(it);
        }
        GroupGraph gg;
        const cudaError_t e = capture_group(ss, n, fields, rhss, types, &gg.exec);
        if (e != cudaSuccess) {
            for (int i = 0; i < n; ++i) ss[i]->last_error = (int)e;
            cudaGetLastError();
            return -4;
        }
        for (int i = 0; i < n; ++i) gg.gens.push_back(ss[i]->gen);
        it = g_groups.emplace(key, gg).first;
    }
    // the members' next host-array solves wait for the caller's stream again
    for (int i = 0; i < n; ++i) ss[i]->cs_follows = false;
    const cudaError_t e = cudaGraphLaunch(it->second.exec, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        for (int i = 0; i < n; ++i) ss[i]->last_error = (int)e;
        return -4;
    }
    return 0;
}
