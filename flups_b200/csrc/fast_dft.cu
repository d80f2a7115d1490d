// Dispatch of the register-resident DFT passes (kernels in fast_dft_impl.cuh,
// instantiated per precision and mode in fast_col_*.cu and fast_row.cu so
// that the units compile in parallel).
#include <cudaTypedefs.h>

#include "fast_dft_impl.cuh"

namespace flb {

// powers of two and 3 x powers of two
bool fast_col_supported(int L) {
    switch (L) {
        case 64: case 128: case 256: case 512: case 1024: case 2048:
        case 48: case 96: case 192: case 384: case 768: case 1536: return true;
    }
    return false;
}
bool fast_row_supported(int L) {
    switch (L) {
        case 64: case 128: case 256: case 512: case 1024: case 2048: case 4096:
        case 48: case 96: case 192: case 384: case 768: case 1536: case 3072: return true;
    }
    return false;
}

int fast_radix1(int f64, int n) { return fast_radix1_of(n, f64); }

int fast_row_tile_rows(int f64, int L) {
    const int lh = L / 2, r1 = fast_radix1_row(lh, f64), p = lh / r1;
    const int threads = (f64 && r1 == 32) ? 128 : 256;
    return p >= threads ? 1 : threads / p;
}

int fast_rowrot_rows(int f64, int L) {
    const int p = L / fast_radix1_rowrot(L, f64);
    return p > 32 ? 0 : FLB_ROWROT_TRIPLES * (32 / p);
}

int fast_col_tile_width(int f64, int L, int tile) {
    const int r1 = fast_radix1_mode(L, f64, 0);
    return col_tile_threads(L, tile, (f64 && L % 3 != 0) || r1 == 48) / (L / r1);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }();
    return fn;
}

bool make_prefetch(Prefetch& pf, const void* base, const uint64_t dims[4], const uint64_t strides[3], const uint32_t box[4],
                   int nbox, int step, int dist) {
    pf.nbox = 0;
    auto fn = tensor_map_encoder();
    if (!fn || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
    cuuint64_t d[4], st[3];
    cuuint32_t b[4], es[4] = {1, 1, 1, 1};
    for (int i = 0; i < 4; ++i) {
        if (dims[i] < 1 || dims[i] > (1ull << 32) || box[i] < 1 || box[i] > 256) return false;
        d[i] = dims[i];
        b[i] = box[i];
    }
    for (int i = 0; i < 3; ++i) {
        if (strides[i] % 16 != 0 || strides[i] >= (1ull << 40)) return false;
        st[i] = strides[i];
    }
    if ((b[0] * 8) % 16 != 0) return false;
    if (fn(&pf.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(base), d, st, b, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    pf.nbox = nbox;
    pf.step = step;
    pf.dist = dist;
    return true;
}

int fast_stage_table_len(int n, int f64) { return stage_table_entries(n, fast_radix1_of(n, f64)); }
int fast_stage_table_len_r1(int n, int r1) { return stage_table_entries(n, r1); }

#ifndef FLB_COL_HALF1
#define FLB_COL_HALF1 1
#endif
cudaError_t launch_fast_col(int f64, int mode, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    auto shape = [L](int n) { return n == L ? SH_FULL : (2 * n == L ? SH_HALF : SH_ANY); };
    int sh;
    if (mode == 0) sh = (a.nout == L) ? shape(a.nin) : SH_ANY;
    else if (mode == 1) sh = (a.nin == L) ? shape(a.nout) : SH_ANY;
    else sh = (shape(a.nin) == shape(a.nout)) ? shape(a.nin) : SH_ANY;
    // fused lines of a node-centred unbounded direction: L/2 + 1 in and out
    if (FLB_COL_HALF1 && mode == 2 && L % 2 == 0 && 2 * a.nin == L + 2 && a.nout == a.nin) sh = SH_HALF1;
    if (mode == 3) return f64 ? launch_col_f64_m3(sh, L, a, ncomp, s) : launch_col_f32_m3(sh, L, a, ncomp, s);
    if (f64) return (mode == 2) ? launch_col_f64_m2(sh, L, a, ncomp, s) : launch_col_f64_m01(mode, sh, L, a, ncomp, s);
    if (mode == 2) return launch_col_f32_m2(sh, L, a, ncomp, s);
    return launch_col_f32_m01(mode, sh, L, a, ncomp, s);
}

bool fast_rowfused_supported(int f64, int L) { return fast_rowfused_len(L, f64); }

cudaError_t launch_fast_rowfused(int f64, int rot, int L, const RowFusedArgs& a, int ncomp, cudaStream_t s) {
    auto shape = [L](int n) { return n == L ? SH_FULL : (2 * n == L ? SH_HALF : SH_ANY); };
    const int sh = (shape(a.nin) == shape(a.nout)) ? shape(a.nin) : SH_ANY;
    if (f64) return launch_rowfused_f64(rot, sh, L, a, ncomp, s);
    return launch_rowfused_f32(rot, sh, L, a, ncomp, s);
}

bool fast_r2r_supported(int M) {
    switch (M) {
        case 64: case 96: case 128: case 192: case 256: case 384: case 512: case 768: case 1024: case 2048: return true;
    }
    return false;
}

#ifndef FLB_DCT1_HALF
#define FLB_DCT1_HALF 1
#endif
static bool dct_len_ok(int n) {
    switch (n) {
        case 64: case 96: case 128: case 192: case 256: case 384: case 512: case 768: case 1024: case 1536: case 2048: return true;
    }
    return false;
}

int fast_dct_length(int kind, int n, int M) { return fast_dct_family(kind, n, M) == 1 ? M : n; }

int fast_dct_family(int kind, int n, int M) {
    // DCT-I / DST-I: the M-point real DFT of the even / odd extension
    if ((kind == LK_DCT1 && M == 2 * (n - 1)) || (kind == LK_DST1 && M == 2 * (n + 1))) return (FLB_DCT1_HALF && dct_len_ok(M)) ? 1 : 0;
    if (M != 2 * n || !dct_len_ok(n)) return 0;
    switch (kind) {
        case LK_DCT2: case LK_DST2: return 2;
        case LK_DCT3: case LK_DST3: return 3;
        case LK_DCT4: case LK_DST4: return 4;
    }
    return 0;
}

cudaError_t launch_fast_r2r(int f64, int M, const RowArgs& a, int ncomp, cudaStream_t s) {
    switch (fast_dct_family(a.kind, a.n, M)) {
        case 1: return launch_dct1_units(f64, a.in_f64, a.out_f64, M, a, ncomp, s);
        case 2: return launch_dct2_units(f64, a.in_f64, a.out_f64, a.n, a, ncomp, s);
        case 3: return launch_dct3_units(f64, a.in_f64, a.out_f64, a.n, a, ncomp, s);
        case 4: return launch_dct4_units(f64, a.in_f64, a.out_f64, a.n, a, ncomp, s);
    }
    return launch_r2r_units(f64, a.in_f64, a.out_f64, M, a, ncomp, s);
}

cudaError_t launch_fast_colreal(int f64, int c2r, int L, const ColArgs& a, int ncomp, cudaStream_t s) {
    auto shape = [L](int n) { return n == L ? SH_FULL : (2 * n == L ? SH_HALF : SH_ANY); };
    // the periodic copy's extra element is stored apart
    const int sh = c2r ? shape(a.period >= 0 ? a.nout - 1 : a.nout) : shape(a.nin > L ? L : a.nin);
    if (f64) return launch_colreal_f64(c2r, sh, L, a, ncomp, s);
    if (a.real64) return launch_colreal_f32u(c2r, sh, L, a, ncomp, s);
    return launch_colreal_f32(c2r, sh, L, a, ncomp, s);
}

// the real side (r2c input / c2r output) is the user's doubles or the working precision
cudaError_t launch_fast_row(int f64, int c2r, int L, const RowArgs& a, int ncomp, cudaStream_t s) {
    const bool half = c2r ? (2 * a.nout == L) : (2 * a.nin == L);
    const int xt64 = c2r ? a.out_f64 : a.in_f64;
    return launch_row_units(f64, c2r, xt64, half, L, a, ncomp, s);
}

}  // namespace flb
