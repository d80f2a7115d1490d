// x and y transforms of one z plane per 16-CTA cluster (FP32, user arrays in
// FP64): the forward kernel does the x r2c rows and the y forward columns of
// the all-unbounded (x, y) pair, the backward kernel the y inverse columns and
// the x c2r rows, with the plane's x spectrum held in the cluster's shared
// memory between the two (distributed shared memory, one transpose through
// the SM-to-SM network) instead of a round trip through HBM.  Same transforms
// and arithmetic as the separate passes (row_r2c_kernel / col_dft_kernel /
// row_c2r_kernel, FFTW_plan_dim.cpp:670-716 in the reference); the spectrum
// column k = LH (the Nyquist column, one value per row) goes through the
// x spectrum array and a one-column launch of the column kernel.
//
// Forward, per plane (cluster rank q of 16):
//   rows    y in [q RPC, (q+1) RPC): load, LH-point DFT of the packed pairs,
//           r2c split; X[k] is stored into the shared memory of the CTA that
//           owns column k (k / CPC), X[LH] into the x spectrum array;
//   barrier (the plane's x spectrum is complete across the cluster);
//   columns k in [q CPC, (q+1) CPC): NY values from own shared memory,
//           2NY-point forward DFT (upper half zero), 2NY outputs to HBM.
// Backward, per plane: columns (2NY values from HBM, inverse DFT, NY outputs
// stored into the row owners' shared memory), barrier, rows (c2r with X[LH]
// from the x spectrum array, LH-point inverse DFT, 2 LH reals to HBM).
// A second cluster barrier per plane keeps the next plane's remote stores
// behind the last local read of the buffer.  Clusters are persistent (one per
// 16 SMs the GPU can co-schedule) and walk the planes.
#include <cstring>

#include "fast_dft_impl.cuh"

namespace flb {

namespace {

constexpr int XY_NC = 16;        // CTAs per cluster
constexpr int XY_THREADS = 256;

template <int LH, int NY>
struct XY {
    using FR = RegFFT<float, LH, 32, true>;  // rows: LH-point DFT of the packed pairs
    using FC = RegFFT<float, 2 * NY, 32>;    // columns: 2NY-point DFT
    static constexpr int PR = FR::P, PC = FC::P;
    static constexpr int RPC = NY / XY_NC;   // rows per CTA (= PC)
    static constexpr int CPC = LH / XY_NC;   // columns per CTA (= 2 PR)
    static constexpr int TRA = XY_THREADS / PR;  // row lines the threads cover
    static constexpr int TR = TRA < RPC ? TRA : RPC;  // rows per round
    static constexpr int TX = XY_THREADS / PC;   // columns per round
    static_assert(PC == RPC && CPC == 2 * PR, "cluster split");
    static_assert(RPC % TR == 0 && CPC % TX == 0 && CPC >= 16, "rounds");
    static_assert(FR::TWS && FC::TWS, "stage tables in shared memory");
    // forward: column buffer [NY][CPC], column c of row y at c ^ 8 (y & 1):
    // the two rows met by a half-warp of the column loads use disjoint banks
    static constexpr int FBUF = NY * CPC;
    // backward: row buffer [RPC][SCB] in the row DFT's line layout (sw(k));
    // the 8-element offset puts consecutive rows on the other 16 banks
    static constexpr int SCB = ((LH + LH / 32 + 15) / 16) * 16 + 8;
    static constexpr int BBUF = RPC * SCB;
    static constexpr int XR = TRA * FR::SC, XC = TX * FC::SC;
    static constexpr int XCH = XR > XC ? XR : XC;  // exchange lines of either phase
    static constexpr int TAB = FR::TW_SMEM + LH + FC::TW_SMEM;
    static constexpr size_t smem(bool fwd) { return (size_t)((fwd ? FBUF : BBUF) + XCH + TAB) * sizeof(float2); }
};

__device__ __forceinline__ uint32_t dsmem_addr(const void* local, int rank) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(local);
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ void dsmem_st(uint32_t addr, float2 v) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
__device__ __forceinline__ void l2_prefetch_bytes(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// the three tables (row stage table, W_L^k for k < LH, column stage table)
template <int LH, int NY>
__device__ __forceinline__ void xy_tables(const XYArgs& a, float2* tab) {
    using X = XY<LH, NY>;
    stage_table_part<float2, X::FR::TW_SMEM>(a.tw_row, tab);
    stage_table_part<float2, LH>(a.tw_split, tab + X::FR::TW_SMEM);
    stage_table_part<float2, X::FC::TW_SMEM>(a.tw_col, tab + X::FR::TW_SMEM + LH);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
}

template <int LH, int NY>
__global__ void __launch_bounds__(XY_THREADS, 1) xy_forward_kernel(const __grid_constant__ XYArgs a) {
    using X = XY<LH, NY>;
    using FR = typename X::FR;
    using FC = typename X::FC;
    using C = float2;
    constexpr int PR = X::PR, PC = X::PC, RPC = X::RPC, CPC = X::CPC, TR = X::TR, TX = X::TX;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* buf = reinterpret_cast<C*>(smraw);
    C* xch = buf + X::FBUF;
    C* tab = xch + X::XCH;
    const C* twr = tab;
    const C* tws = tab + FR::TW_SMEM;
    const C* twc = tab + FR::TW_SMEM + LH;
    const int q = (int)(blockIdx.x % XY_NC), cid = (int)(blockIdx.x / XY_NC), ncl = (int)(gridDim.x / XY_NC);
    const int tid = threadIdx.x;
    const int nplanes = a.nz * a.ncomp;
    xy_tables<LH, NY>(a, tab);
    // every CTA of the cluster is running before the first remote store
    cluster_arrive();
    cluster_wait();
    // row phase lanes
    const int pr = tid % PR, rr = tid / PR;
    const bool ract = rr < TR;
    // column phase lanes; the swizzle of the column buffer depends on y & 1 = p & 1
    const int cc0 = tid % TX, pc = tid / TX;
    const int csw = (pc & 1) << 3;
    bool pending = false;  // an arrive (buffer read) waits for its wait
    for (int pl = cid; pl < nplanes; pl += ncl) {
        const int comp = pl / a.nz, z = pl % a.nz;
        const double* uin = reinterpret_cast<const double*>(a.in) + comp * a.u_cstr + (int64_t)z * a.u_s2;
        if (pending) cluster_wait();  // every CTA has read its buffer of the previous plane
        pending = false;
        // ---------------- rows: x r2c
#pragma unroll 1
        for (int rd = 0; rd < RPC / TR; ++rd) {
            const int y = q * RPC + rd * TR + (ract ? rr : 0);
            const double* src = uin + (int64_t)y * a.u_s1 + 2 * pr;
            C v[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                if (r >= 16) {
                    v[r] = mkc(0.f, 0.f);
                } else {
                    const double2 d = *reinterpret_cast<const double2*>(src + 2 * PR * r);
                    v[r] = mkc((float)d.x, (float)d.y);
                }
            }
            C* line = xch + rr * FR::SC;
            FR::template fft<true, false>(v, line, pr, twr);
            // X[k] = 1/2 (Z_k + conj Z_{LH-k}) - i/2 W_L^k (Z_k - conj Z_{LH-k}),  Z_LH = Z_0
            __syncthreads();
#pragma unroll
            for (int r = 0; r < 32; ++r) line[FR::sw(pr + PR * r)] = v[r];
            __syncthreads();
            if (ract) {
                const C* tw = tws + pr;
                const int ysw = (y & 1) << 3;
#pragma unroll
                for (int r = 0; r < 32; ++r) {
                    const int k = pr + PR * r;
                    const C zk = v[r];
                    const C zm = cconj(line[FR::sw(k == 0 ? 0 : LH - k)]);
                    const C e = cadd(zk, zm);
                    const C d = csub(zk, zm);
                    const C w = cmul(tw[PR * r], d);
                    const C xk = mkc(0.5f * (e.x + w.y), 0.5f * (e.y - w.x));
                    // owner r / 2, column pr + PR (r & 1) of its buffer
                    const int col = pr + PR * (r & 1);
                    dsmem_st(dsmem_addr(buf + y * CPC + (col ^ ysw), r >> 1), xk);
                }
                if (pr == 0) {
                    const C z0 = line[0];
                    reinterpret_cast<C*>(a.nyq)[comp * a.n_c + (int64_t)z * a.n_s2 + (int64_t)y * a.n_s1] = mkc(z0.x - z0.y, 0.f);
                }
            }
        }
        // the plane's x spectrum is complete in the cluster's buffers
        cluster_arrive();
        cluster_wait();
        // the rows of this CTA in the plane it does next: into L2 while the columns run
        if (a.prefetch && tid < RPC && pl + ncl < nplanes) {
            const int pn = pl + ncl, cn = pn / a.nz, zn = pn % a.nz;
            l2_prefetch_bytes(reinterpret_cast<const double*>(a.in) + cn * a.u_cstr + (int64_t)zn * a.u_s2 +
                                  (int64_t)(q * RPC + tid) * a.u_s1,
                              LH * 8);
        }
        // ---------------- columns: y forward
        C* outp = reinterpret_cast<C*>(a.out) + comp * a.s_c + (int64_t)z * a.s_o;
#pragma unroll 1
        for (int cr = 0; cr < CPC / TX; ++cr) {
            const int cc = cr * TX + cc0;
            C v[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) v[r] = (r < 16) ? buf[(pc + PC * r) * CPC + (cc ^ csw)] : mkc(0.f, 0.f);
            if (cr == CPC / TX - 1) {
                cluster_arrive();  // this CTA's buffer is read: the next plane's rows may overwrite it
                pending = true;
            }
            FC::template fft<true, false>(v, xch + cc0 * FC::SC, pc, twc);
            C* o = outp + (int64_t)pc * a.s_l + q * CPC + cc;
            const int os = PC * (int)a.s_l;
#pragma unroll
            for (int r = 0; r < 32; ++r) o[r * os] = v[r];
        }
    }
    if (pending) cluster_wait();
}

template <int LH, int NY>
__global__ void __launch_bounds__(XY_THREADS, 1) xy_backward_kernel(const __grid_constant__ XYArgs a) {
    using X = XY<LH, NY>;
    using FR = typename X::FR;
    using FC = typename X::FC;
    using C = float2;
    constexpr int PR = X::PR, PC = X::PC, RPC = X::RPC, CPC = X::CPC, TR = X::TR, TX = X::TX, SCB = X::SCB;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* buf = reinterpret_cast<C*>(smraw);
    C* xch = buf + X::BBUF;
    C* tab = xch + X::XCH;
    const C* twr = tab;
    const C* tws = tab + FR::TW_SMEM;
    const C* twc = tab + FR::TW_SMEM + LH;
    const int q = (int)(blockIdx.x % XY_NC), cid = (int)(blockIdx.x / XY_NC), ncl = (int)(gridDim.x / XY_NC);
    const int tid = threadIdx.x;
    const int nplanes = a.nz * a.ncomp;
    xy_tables<LH, NY>(a, tab);
    cluster_arrive();
    cluster_wait();
    const int cc0 = tid % TX, pc = tid / TX;
    const int pr = tid % PR, rr = tid / PR;
    const bool ract = rr < TR;
    bool pending = false;
    for (int pl = cid; pl < nplanes; pl += ncl) {
        const int comp = pl / a.nz, z = pl % a.nz;
        // ---------------- columns: y inverse, the kept half to the row owners
        const C* inp = reinterpret_cast<const C*>(a.in) + comp * a.s_c + (int64_t)z * a.s_o;
        if (pending) cluster_wait();  // every CTA's rows of the previous plane are done with its buffer
        pending = false;
#pragma unroll 1
        for (int cr = 0; cr < CPC / TX; ++cr) {
            const int kx = q * CPC + cr * TX + cc0;
            const C* src = inp + (int64_t)pc * a.s_l + kx;
            const int ls = PC * (int)a.s_l;
            C v[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) v[r] = src[r * ls];
            FC::template fft<false, true>(v, xch + cc0 * FC::SC, pc, twc);
            // y = pc + PC r < NY: owner r, its row pc
            C* dl = buf + pc * SCB + FR::sw(kx);
#pragma unroll
            for (int r = 0; r < 16; ++r) dsmem_st(dsmem_addr(dl, r), v[r]);
        }
        cluster_arrive();
        cluster_wait();
        // the columns of this CTA in the plane it does next: into L2 while the rows run
        if (a.prefetch && pl + ncl < nplanes) {
            const int pn = pl + ncl, cn = pn / a.nz, zn = pn % a.nz;
            const C* nb = reinterpret_cast<const C*>(a.in) + cn * a.s_c + (int64_t)zn * a.s_o + q * CPC;
            for (int ky = tid; ky < 2 * NY; ky += XY_THREADS) l2_prefetch_bytes(nb + (int64_t)ky * a.s_l, CPC * 8);
        }
        // ---------------- rows: x c2r
        double* uout = reinterpret_cast<double*>(a.out) + comp * a.u_cstr + (int64_t)z * a.u_s2;
#pragma unroll 1
        for (int rd = 0; rd < RPC / TR; ++rd) {
            const int yl = rd * TR + (ract ? rr : 0);
            const int y = q * RPC + yl;
            // lanes past the CTA's rows work on a scratch line and store nothing
            C* line = ract ? buf + yl * SCB : xch + (rr - TR) * FR::SC;
            const C xl = reinterpret_cast<const C*>(a.nyq)[comp * a.n_c + (int64_t)z * a.n_s2 + (int64_t)y * a.n_s1];
            // Z'_k = A_k + i B_k, A = X_k + conj X_{LH-k}, B = (X_k - conj X_{LH-k}) W_L^{-k}
            const C* tw = tws + pr;
            C v[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                const int k = pr + PR * r;
                C xk = line[FR::sw(k)];
                C xm = line[FR::sw(k == 0 ? 0 : LH - k)];
                if (k == 0) {
                    xm = xl;
                    xk.y = 0.f;
                    xm.y = 0.f;
                }
                xm = cconj(xm);
                const C A = cadd(xk, xm);
                const C B = cmul(csub(xk, xm), cconj(tw[PR * r]));
                v[r] = mkc(A.x - B.y, A.y + B.x);
            }
            FR::template fft<false, true>(v, line, pr, twr);
            if (rd == RPC / TR - 1) {
                cluster_arrive();  // this CTA's buffer is read: the next plane's columns may overwrite it
                pending = true;
            }
            if (ract) {
                double* dst = uout + (int64_t)y * a.u_s1 + 2 * pr;
#pragma unroll
                for (int r = 0; r < 16; ++r) *reinterpret_cast<double2*>(dst + 2 * PR * r) = make_double2((double)v[r].x, (double)v[r].y);
            }
        }
    }
    if (pending) cluster_wait();
}

template <typename K>
cudaError_t xy_config(K kernel, size_t smem, std::atomic<unsigned long long>& attr, cudaLaunchConfig_t& cfg,
                      cudaLaunchAttribute* at, cudaStream_t s) {
    int dev = 0;
    if (cudaError_t e = cudaGetDevice(&dev); e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr.load(std::memory_order_acquire) & bit)) {
        if (cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); e != cudaSuccess)
            return e;
        if (cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1); e != cudaSuccess)
            return e;
        attr.fetch_or(bit, std::memory_order_acq_rel);
    }
    memset(&cfg, 0, sizeof(cfg));
    cfg.blockDim = dim3(XY_THREADS, 1, 1);
    cfg.gridDim = dim3(XY_NC, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = XY_NC;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaSuccess;
}

template <int LH, int NY, bool FWD>
cudaError_t xy_launch_t(const XYArgs* a, int* nclusters, cudaStream_t s) {
    using X = XY<LH, NY>;
    auto kernel = FWD ? xy_forward_kernel<LH, NY> : xy_backward_kernel<LH, NY>;
    const size_t smem = X::smem(FWD);
    static std::atomic<unsigned long long> attr{0};
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at[1];
    if (cudaError_t e = xy_config(kernel, smem, attr, cfg, at, s); e != cudaSuccess) return e;
    int n = 0;
    if (cudaError_t e = cudaOccupancyMaxActiveClusters(&n, kernel, &cfg); e != cudaSuccess) return e;
    if (nclusters) *nclusters = n;
    if (!a) return cudaSuccess;
    if (n < 1) return cudaErrorInvalidConfiguration;
    const int planes = a->nz * a->ncomp;
    const int ncl = planes < n ? planes : n;
    cfg.gridDim = dim3(XY_NC * ncl, 1, 1);
    return cudaLaunchKernelEx(&cfg, kernel, *a);
}

}  // namespace

bool xy_cluster_supported(int LH, int NY) { return (LH == 512 && NY == 512) || (LH == 256 && NY == 256); }

size_t xy_cluster_smem(int fwd, int LH, int NY) {
    if (LH == 512 && NY == 512) return XY<512, 512>::smem(fwd != 0);
    if (LH == 256 && NY == 256) return XY<256, 256>::smem(fwd != 0);
    return 0;
}

cudaError_t launch_xy_cluster(int fwd, int LH, int NY, const XYArgs* a, int* nclusters, cudaStream_t s) {
    if (LH == 512 && NY == 512) return fwd ? xy_launch_t<512, 512, true>(a, nclusters, s) : xy_launch_t<512, 512, false>(a, nclusters, s);
    if (LH == 256 && NY == 256) return fwd ? xy_launch_t<256, 256, true>(a, nclusters, s) : xy_launch_t<256, 256, false>(a, nclusters, s);
    return cudaErrorInvalidValue;
}

}  // namespace flb
