// Lattice Green's function tables and far-field expansions.
//
// Tables: raw little-endian doubles, 32^3 (3-D) or 32^2 (2-D), index
// ix + iy N + iz N^2, the reference's kernel/*.ker files (file names as in
// src/green_functions.hpp:53-72).  They are looked up next to this library
// (<dir of libflups_b200.so>/kernel), or in $FLUPS_KERNEL_PATH.
// Far-field expansions: coefficient tables generated from
// flups_b200/kernel/farfield.json at build time (farfield_data.inc).
#include <dlfcn.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "host.hpp"

namespace {
struct FarTable {
    const char* name;
    int ndim;
    int nterms;
    const double* coef;  // already multiplied by pi^p
    const int* exps;     // a, b, c, e per term
    double logc;
};
#include "farfield_data.inc"

std::string kernel_dir() {
    if (const char* e = getenv("FLUPS_KERNEL_PATH")) return std::string(e);
    Dl_info info;
    if (dladdr((void*)&kernel_dir, &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        const size_t s = p.find_last_of('/');
        if (s != std::string::npos) return p.substr(0, s) + "/kernel";
    }
    return "kernel";
}
}  // namespace

namespace flb {

int load_lgf_table(int kind, int ndim, std::vector<double>& data) {
    int order = 0;
    if (kind == LGF_2) order = 2;
    else if (kind == LGF_4 || kind == MEHR_4L || kind == MEHR_4F) order = 4;
    else if (kind == LGF_6 || kind == MEHR_6L || kind == MEHR_6F) order = 6;
    else if (kind == LGF_8) order = 8;
    FLB_CHECK(order > 0, "LGF Kernel type not recognized");
    const int N = 32;
    char name[64];
    if (ndim == 3) {
        if (kind == MEHR_4L || kind == MEHR_6L) snprintf(name, sizeof(name), "MEHR_%dL_3d_%d.ker", order, N);
        else if (kind == MEHR_4F || kind == MEHR_6F) snprintf(name, sizeof(name), "MEHR_%dF_3d_%d.ker", order, N);
        else snprintf(name, sizeof(name), "LGF_%d_3d_%d.ker", order, N);
    } else {
        if (kind == MEHR_4L || kind == MEHR_6L) snprintf(name, sizeof(name), "MEHR_4L6L_2d_%d.ker", N);
        else if (kind == MEHR_4F || kind == MEHR_6F) snprintf(name, sizeof(name), "MEHR_%dF_2d_%d.ker", order, N);
        else snprintf(name, sizeof(name), "LGF_%d_2d_%d.ker", order, N);
    }
    const std::string path = kernel_dir() + "/" + name;
    const size_t count = (ndim == 3) ? (size_t)N * N * N : (size_t)N * N;
    data.assign(count, 0.0);
    FILE* f = fopen(path.c_str(), "rb");
    FLB_CHECK(f != nullptr, "unable to read file %s", path.c_str());
    const size_t got = fread(data.data(), sizeof(double), count, f);
    fclose(f);
    FLB_CHECK(got == count, "short LGF table %s", path.c_str());
    return N;
}

int farfield_terms(int kind, int ndim, std::vector<FarTerm>& terms, double& logc) {
    const char* base = nullptr;
    switch (kind) {
        case LGF_2: base = "lgf_2"; break;
        case LGF_4: base = "lgf_4"; break;
        case LGF_6: base = "lgf_6"; break;
        case LGF_8: base = "lgf_8"; break;
        case MEHR_4L: base = (ndim == 2) ? "mehr_4l6l" : "mehr_4l"; break;
        case MEHR_6L: base = (ndim == 2) ? "mehr_4l6l" : "mehr_6l"; break;
        case MEHR_4F: base = "mehr_4f"; break;
        case MEHR_6F: base = "mehr_6f"; break;
    }
    FLB_CHECK(base != nullptr, "no far-field expansion for kernel %d", kind);
    char name[64];
    snprintf(name, sizeof(name), "%s_%dunb0spe", base, ndim);
    for (const FarTable& t : kFarTables) {
        if (strcmp(t.name, name) != 0) continue;
        terms.resize(t.nterms);
        for (int i = 0; i < t.nterms; ++i) {
            terms[i].coef = t.coef[i];
            terms[i].a = t.exps[4 * i];
            terms[i].b = t.exps[4 * i + 1];
            terms[i].c = t.exps[4 * i + 2];
            terms[i].e = t.exps[4 * i + 3];
        }
        logc = t.logc;
        return t.nterms;
    }
    FLB_CHECK(false, "far-field table %s missing", name);
    return 0;
}

}  // namespace flb
