// FP64 FFT behind the FFTW-API subset of fftw3.h in this directory, so that
// the reference's solver sources compile and run without FFTW.  Test
// infrastructure of the oracle: checked against scipy.fft (pocketfft) by
// tests/test_oracle_ref_build.py before the reference build it serves is
// trusted.
//
// Conventions are FFTW 3.3's (unnormalised transforms):
//   DFT       Y_k = sum_j X_j exp(s 2 pi i j k / n), s = sign (-1 forward)
//   r2c       the first n/2 + 1 outputs of the forward DFT of a real row
//   c2r       the real backward DFT of a Hermitian half spectrum (n/2 + 1
//             inputs; imaginary parts of the 0 and n/2 modes ignored)
//   REDFT00   Y_k = X_0 + (-1)^k X_{n-1} + 2 sum_{j=1}^{n-2} X_j cos(pi j k / (n-1))
//   REDFT10   Y_k = 2 sum_j X_j cos(pi (j + 1/2) k / n)
//   REDFT01   Y_k = X_0 + 2 sum_{j>=1} X_j cos(pi j (k + 1/2) / n)
//   REDFT11   Y_k = 2 sum_j X_j cos(pi (j + 1/2) (k + 1/2) / n)
//   RODFT00   Y_k = 2 sum_j X_j sin(pi (j + 1) (k + 1) / (n + 1))
//   RODFT10   Y_k = 2 sum_j X_j sin(pi (j + 1/2) (k + 1) / n)
//   RODFT01   Y_k = (-1)^k X_{n-1} + 2 sum_{j<n-1} X_j sin(pi (j + 1) (k + 1/2) / n)
//   RODFT11   Y_k = 2 sum_j X_j sin(pi (j + 1/2) (k + 1/2) / n)
// Each r2r kind is the real or imaginary part of one complex DFT of a
// symmetric extension of the row (length 2(n-1), 2(n+1), 4n or 8n), placed
// so that the wanted cosine or sine sum is a DFT output (derivations beside
// each case below).  The complex DFT is a mixed-radix Stockham transform
// (radices 2, 3, 4, 5 and any other small prime by direct sums) and
// Bluestein's chirp convolution for lengths with a prime factor above 13.
// Rank-0 guru plans over two "howmany" dimensions are the strided copies
// (transposes) the reference uses to reorder its pencils.
#include <stdint.h>
#include <string.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "fftw3.h"

namespace {

using cd = std::complex<double>;

// exp(s 2 pi i t / n) for t = 0..n-1, computed in long double
std::vector<cd> roots(int n, int s) {
    std::vector<cd> w(n);
    const long double two_pi = 6.283185307179586476925286766559L;
    for (int t = 0; t < n; ++t) {
        const long double a = two_pi * (long double)t / (long double)n;
        w[t] = cd((double)cosl(a), (double)(s * sinl(a)));
    }
    return w;
}

struct Cfft {
    int n = 1, s = -1;
    std::vector<int> radix;  // Stockham stages, first to last
    std::vector<cd> w;       // exp(s 2 pi i t / n)
    // Bluestein
    bool blue = false;
    int m = 0;
    std::vector<cd> chirp;  // exp(s pi i j^2 / n), j < n
    std::vector<cd> bhat;   // DFT_m of the conjugate chirp, wrapped
    std::unique_ptr<Cfft> fwd, bwd;

    Cfft(int n_, int s_) : n(n_), s(s_) {
        int r = n, maxp = 1;
        std::vector<int> f;
        while (r % 4 == 0) { f.push_back(4); r /= 4; }
        while (r % 2 == 0) { f.push_back(2); r /= 2; }
        for (int p = 3; r > 1; p += 2) {
            while (r % p == 0) { f.push_back(p); r /= p; maxp = p > maxp ? p : maxp; }
            if ((long long)p * p > r && r > 1) { f.push_back(r); maxp = r > maxp ? r : maxp; r = 1; }
        }
        if (maxp > 13) {
            blue = true;
            m = 1;
            while (m < 2 * n - 1) m <<= 1;
            chirp.resize(n);
            const long double pi = 3.141592653589793238462643383279L;
            for (int j = 0; j < n; ++j) {
                const long long q = ((long long)j * j) % (2LL * n);  // j^2 mod 2n keeps the angle exact
                const long double a = pi * (long double)q / (long double)n;
                chirp[j] = cd((double)cosl(a), (double)(s * sinl(a)));
            }
            fwd.reset(new Cfft(m, -1));
            bwd.reset(new Cfft(m, +1));
            std::vector<cd> b(m, cd(0, 0)), tmp(m);
            for (int j = 0; j < n; ++j) {
                b[j] = std::conj(chirp[j]);
                if (j > 0) b[m - j] = std::conj(chirp[j]);
            }
            fwd->run(b.data(), tmp.data());
            bhat = b;
        } else {
            radix = f;
            w = roots(n, s);
        }
    }

    // direct sum for a small radix p: the p-th roots are w[t n / p]
    void dft_small(cd* v, int p) const {
        cd out[64];
        const int q = n / p;
        for (int k = 0; k < p; ++k) {
            cd acc(0, 0);
            for (int j = 0; j < p; ++j) acc += v[j] * w[(size_t)((j * k) % p) * q];
            out[k] = acc;
        }
        for (int k = 0; k < p; ++k) v[k] = out[k];
    }

    // in-place butterflies of radix p (unnormalised DFT of sign s)
    void bfly(cd* v, int p) const {
        const double sg = (double)s;
        if (p == 2) {
            const cd a = v[0], b = v[1];
            v[0] = a + b;
            v[1] = a - b;
        } else if (p == 4) {
            const cd a = v[0] + v[2], b = v[0] - v[2], c = v[1] + v[3], d = v[1] - v[3];
            const cd jd(-sg * d.imag(), sg * d.real());  // (s i) d
            v[0] = a + c;
            v[2] = a - c;
            v[1] = b + jd;
            v[3] = b - jd;
        } else if (p == 3) {
            const double c3 = -0.5, s3 = sg * 0.86602540378443864676;
            const cd a = v[0], b = v[1], c = v[2];
            const cd t = b + c, u = b - c;
            const cd m1 = a + c3 * t, m2(-s3 * u.imag(), s3 * u.real());
            v[0] = a + t;
            v[1] = m1 + m2;
            v[2] = m1 - m2;
        } else {
            dft_small(v, p);
        }
    }

    // x (length n) transformed in place; work: n entries of scratch
    void run(cd* x, cd* work) const {
        if (n == 1) return;
        if (blue) {
            std::vector<cd> a(m, cd(0, 0)), t(m);
            for (int j = 0; j < n; ++j) a[j] = x[j] * chirp[j];
            fwd->run(a.data(), t.data());
            for (int k = 0; k < m; ++k) a[k] *= bhat[k];
            bwd->run(a.data(), t.data());
            const double inv = 1.0 / (double)m;
            for (int k = 0; k < n; ++k) x[k] = a[k] * chirp[k] * inv;
            return;
        }
        cd* src = x;
        cd* dst = work;
        int ns = 1;  // length of the sub-transforms already done
        for (int p : radix) {
            const int np = n / p, step = n / (ns * p);
            cd v[64];
            for (int j = 0; j < np; ++j) {
                const int k = j % ns;
                for (int r = 0; r < p; ++r) v[r] = src[j + r * np];
                if (ns > 1)
                    for (int r = 1; r < p; ++r) v[r] *= w[((long long)r * k * step) % n];
                bfly(v, p);
                const int base = (j / ns) * ns * p + k;
                for (int r = 0; r < p; ++r) dst[base + r * ns] = v[r];
            }
            std::swap(src, dst);
            ns *= p;
        }
        if (src != x) memcpy(x, src, sizeof(cd) * n);
    }
};

enum Kind { K_DFT, K_R2C, K_C2R, K_R2R, K_COPY, K_COPYC };

}  // namespace

struct fftw_plan_s {
    Kind kind;
    int n = 0, sign = -1;
    fftw_r2r_kind rk = FFTW_REDFT00;
    int istride = 1, ostride = 1;
    std::unique_ptr<Cfft> f;  // the complex DFT the transform runs on
    int N = 0;                // its length
    std::vector<cd> wr;       // r2c / c2r split factors exp(-+ 2 pi i k / n)
    fftw_iodim hd[2];         // rank-0 copies: the two howmany dimensions
    void* in = nullptr;
    void* out = nullptr;
};

namespace {

// per-thread scratch
std::vector<cd>& scratch(int which, size_t n) {
    thread_local std::vector<cd> buf[3];
    if (buf[which].size() < n) buf[which].resize(n);
    return buf[which];
}

fftw_plan make(Kind k) { return new fftw_plan_s{k}; }

void exec_dft(const fftw_plan p, const double* in, double* out) {
    const int n = p->n;
    std::vector<cd>& x = scratch(0, n);
    std::vector<cd>& wk = scratch(1, n);
    for (int j = 0; j < n; ++j) x[j] = cd(in[2 * (size_t)j * p->istride], in[2 * (size_t)j * p->istride + 1]);
    p->f->run(x.data(), wk.data());
    for (int k = 0; k < n; ++k) {
        out[2 * (size_t)k * p->ostride] = x[k].real();
        out[2 * (size_t)k * p->ostride + 1] = x[k].imag();
    }
}

// r2c: z_j = x_{2j} + i x_{2j+1} (h = n/2 points), Z = DFT_h(z);
// X_k = E_k + exp(-2 pi i k/n) O_k with E_k = (Z_k + conj Z_{h-k}) / 2 and
// O_k = (Z_k - conj Z_{h-k}) / (2i), Z_h = Z_0.  Odd n: the complex DFT of
// the row.
void exec_r2c(const fftw_plan p, const double* in, double* out) {
    const int n = p->n;
    if (n % 2 == 0) {
        const int h = n / 2;
        std::vector<cd>& z = scratch(0, h + 1);
        std::vector<cd>& wk = scratch(1, h);
        for (int j = 0; j < h; ++j) z[j] = cd(in[2 * j], in[2 * j + 1]);
        p->f->run(z.data(), wk.data());
        z[h] = z[0];
        std::vector<cd>& X = scratch(2, h + 1);
        for (int k = 0; k <= h; ++k) {
            const cd a = z[k], b = std::conj(z[h - k]);
            const cd e = 0.5 * (a + b), o = cd(0, -0.5) * (a - b);
            X[k] = e + p->wr[k] * o;
        }
        for (int k = 0; k <= h; ++k) {
            out[2 * k] = X[k].real();
            out[2 * k + 1] = X[k].imag();
        }
    } else {
        std::vector<cd>& x = scratch(0, n);
        std::vector<cd>& wk = scratch(1, n);
        for (int j = 0; j < n; ++j) x[j] = cd(in[j], 0.0);
        p->f->run(x.data(), wk.data());
        for (int k = 0; k <= n / 2; ++k) {
            out[2 * k] = x[k].real();
            out[2 * k + 1] = x[k].imag();
        }
    }
}

// c2r (even n): the inverse of the r2c split above with s = +1:
// Z_k = (X_k + conj X_{h-k}) + i exp(2 pi i k/n) (X_k - conj X_{h-k}), then
// z = the backward DFT_h of Z and x_{2j} = Re z_j, x_{2j+1} = Im z_j.
// Odd n: the backward complex DFT of the Hermitian extension.
void exec_c2r(const fftw_plan p, const double* in, double* out) {
    const int n = p->n;
    const int h = n / 2;
    std::vector<cd>& X = scratch(2, h + 1);
    for (int k = 0; k <= h; ++k) X[k] = cd(in[2 * k], in[2 * k + 1]);
    X[0] = cd(X[0].real(), 0.0);
    if (n % 2 == 0) {
        X[h] = cd(X[h].real(), 0.0);
        std::vector<cd>& z = scratch(0, h);
        std::vector<cd>& wk = scratch(1, h);
        for (int k = 0; k < h; ++k) {
            const cd a = X[k], b = std::conj(X[h - k]);
            z[k] = (a + b) + cd(0, 1) * p->wr[k] * (a - b);
        }
        p->f->run(z.data(), wk.data());
        for (int j = 0; j < h; ++j) {
            out[2 * j] = z[j].real();
            out[2 * j + 1] = z[j].imag();
        }
    } else {
        std::vector<cd>& x = scratch(0, n);
        std::vector<cd>& wk = scratch(1, n);
        for (int k = 0; k <= h; ++k) x[k] = X[k];
        for (int k = h + 1; k < n; ++k) x[k] = std::conj(X[n - k]);
        p->f->run(x.data(), wk.data());
        for (int j = 0; j < n; ++j) out[j] = x[j].real();
    }
}

void exec_r2r(const fftw_plan p, const double* in, double* out) {
    const int n = p->n, N = p->N;
    std::vector<double> X(n);
    for (int j = 0; j < n; ++j) X[j] = in[(size_t)j * p->istride];
    std::vector<cd>& v = scratch(0, N);
    std::vector<cd>& wk = scratch(1, N);
    for (int t = 0; t < N; ++t) v[t] = cd(0, 0);
    std::vector<double> Y(n);
    switch (p->rk) {
        case FFTW_REDFT00:
            // even extension of period 2(n-1): V_k = X_0 + (-1)^k X_{n-1} + 2 sum X_j cos(2 pi j k / N)
            for (int j = 0; j < n; ++j) v[j] = X[j];
            for (int j = 1; j < n - 1; ++j) v[N - j] = X[j];
            p->f->run(v.data(), wk.data());
            for (int k = 0; k < n; ++k) Y[k] = v[k].real();
            break;
        case FFTW_RODFT00:
            // odd extension of period 2(n+1): V_{k+1} = -2i sum X_j sin(pi (j+1)(k+1)/(n+1))
            for (int j = 0; j < n; ++j) {
                v[j + 1] = X[j];
                v[N - j - 1] = -X[j];
            }
            p->f->run(v.data(), wk.data());
            for (int k = 0; k < n; ++k) Y[k] = -v[k + 1].imag();
            break;
        case FFTW_REDFT10:
            // N = 4n, X_j at the odd points 2j+1 and 4n-2j-1: V_k = 2 sum X_j cos(pi (2j+1) k / 2n)
            for (int j = 0; j < n; ++j) {
                v[2 * j + 1] = X[j];
                v[N - 2 * j - 1] = X[j];
            }
            p->f->run(v.data(), wk.data());
            for (int k = 0; k < n; ++k) Y[k] = v[k].real();
            break;
        case FFTW_RODFT10:
            // N = 4n, odd pairs: V_{k+1} = -2i sum X_j sin(pi (2j+1)(k+1) / 2n)
            for (int j = 0; j < n; ++j) {
                v[2 * j + 1] = X[j];
                v[N - 2 * j - 1] = -X[j];
            }
            p->f->run(v.data(), wk.data());
            for (int k = 0; k < n; ++k) Y[k] = -v[k + 1].imag();
            break;
        case FFTW_REDFT01:
            // N = 4n, X_j at j and 4n-j (X_0 once): V_{2k+1} = X_0 + 2 sum X_j cos(pi j (2k+1) / 2n)
            v[0] = X[0];
            for (int j = 1; j < n; ++j) {
                v[j] = X[j];
                v[N - j] = X[j];
            }
            p->f->run(v.data(), wk.data());
            for (int k = 0; k < n; ++k) Y[k] = v[2 * k + 1].real();
            break;
        case FFTW_RODFT01:
            // N = 4n, X_j at j+1 and -X_j at 4n-j-1 for j < n-1, X_{n-1} once at n:
            // V_{2k+1} = -i [(-1)^k X_{n-1} + 2 sum_{j<n-1} X_j sin(pi (j+1)(2k+1) / 2n)]
            for (int j = 0; j < n; ++j) v[j + 1] = X[j];
            for (int j = 0; j < n - 1; ++j) v[N - j - 1] = -X[j];
            p->f->run(v.data(), wk.data());
            for (int k = 0; k < n; ++k) Y[k] = -v[2 * k + 1].imag();
            break;
        case FFTW_REDFT11:
            // N = 8n, X_j at 2j+1 and 8n-2j-1: V_{2k+1} = 2 sum X_j cos(pi (2j+1)(2k+1) / 4n)
            for (int j = 0; j < n; ++j) {
                v[2 * j + 1] = X[j];
                v[N - 2 * j - 1] = X[j];
            }
            p->f->run(v.data(), wk.data());
            for (int k = 0; k < n; ++k) Y[k] = v[2 * k + 1].real();
            break;
        case FFTW_RODFT11:
            for (int j = 0; j < n; ++j) {
                v[2 * j + 1] = X[j];
                v[N - 2 * j - 1] = -X[j];
            }
            p->f->run(v.data(), wk.data());
            for (int k = 0; k < n; ++k) Y[k] = -v[2 * k + 1].imag();
            break;
        default:
            std::fprintf(stderr, "fft shim: r2r kind %d not provided\n", (int)p->rk);
            std::abort();
    }
    for (int k = 0; k < n; ++k) out[(size_t)k * p->ostride] = Y[k];
}

// the strided copy of a rank-0 plan: out[i0 os0 + i1 os1] = in[i0 is0 + i1 is1]
// (elements of w doubles); the input span is read whole first (in place)
void exec_copy(const fftw_plan p, const double* in, double* out, int w) {
    const fftw_iodim a = p->hd[0], b = p->hd[1];
    const size_t span = (size_t)(a.n - 1) * a.is + (size_t)(b.n - 1) * b.is + 1;
    std::vector<double> tmp(span * w);
    memcpy(tmp.data(), in, sizeof(double) * span * w);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) if (!omp_in_parallel())
#endif
    for (int i1 = 0; i1 < b.n; ++i1)
        for (int i0 = 0; i0 < a.n; ++i0)
            for (int e = 0; e < w; ++e)
                out[((size_t)i0 * a.os + (size_t)i1 * b.os) * w + e] = tmp[((size_t)i0 * a.is + (size_t)i1 * b.is) * w + e];
}

int r2r_len(fftw_r2r_kind k, int n) {
    switch (k) {
        case FFTW_REDFT00: return 2 * (n - 1);
        case FFTW_RODFT00: return 2 * (n + 1);
        case FFTW_REDFT10: case FFTW_RODFT10: case FFTW_REDFT01: case FFTW_RODFT01: return 4 * n;
        case FFTW_REDFT11: case FFTW_RODFT11: return 8 * n;
        default: return 0;
    }
}

}  // namespace

extern "C" {

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned) {
    fftw_plan p = make(K_DFT);
    p->n = n;
    p->sign = sign;
    p->f.reset(new Cfft(n, sign));
    p->in = in;
    p->out = out;
    return p;
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned) {
    fftw_plan p = make(K_R2C);
    p->n = n;
    if (n % 2 == 0) {
        p->f.reset(new Cfft(n / 2, -1));
        p->wr = roots(n, -1);
    } else {
        p->f.reset(new Cfft(n, -1));
    }
    p->in = in;
    p->out = out;
    return p;
}

fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex* in, double* out, unsigned) {
    fftw_plan p = make(K_C2R);
    p->n = n;
    if (n % 2 == 0) {
        p->f.reset(new Cfft(n / 2, +1));
        p->wr = roots(n, +1);
    } else {
        p->f.reset(new Cfft(n, +1));
    }
    p->in = in;
    p->out = out;
    return p;
}

fftw_plan fftw_plan_r2r_1d(int n, double* in, double* out, fftw_r2r_kind kind, unsigned) {
    fftw_plan p = make(K_R2R);
    p->n = n;
    p->rk = kind;
    p->N = r2r_len(kind, n);
    if (p->N <= 0 || (kind == FFTW_REDFT00 && n < 2)) {
        std::fprintf(stderr, "fft shim: r2r kind %d of length %d not provided\n", (int)kind, n);
        std::abort();
    }
    p->f.reset(new Cfft(p->N, -1));
    p->in = in;
    p->out = out;
    return p;
}

fftw_plan fftw_plan_many_r2r(int rank, const int* n, int howmany, double* in, const int*, int istride, int, double* out,
                             const int*, int ostride, int, const fftw_r2r_kind* kind, unsigned flags) {
    if (rank != 1 || howmany != 1) {
        std::fprintf(stderr, "fft shim: many_r2r of rank %d, howmany %d not provided\n", rank, howmany);
        std::abort();
    }
    fftw_plan p = fftw_plan_r2r_1d(n[0], in, out, kind[0], flags);
    p->istride = istride;
    p->ostride = ostride;
    return p;
}

static fftw_plan guru_copy(int rank, int howmany_rank, const fftw_iodim* hd, void* in, void* out, Kind k) {
    if (rank != 0 || howmany_rank != 2) {
        std::fprintf(stderr, "fft shim: guru plan of rank %d over %d dimensions not provided\n", rank, howmany_rank);
        std::abort();
    }
    fftw_plan p = make(k);
    p->hd[0] = hd[0];
    p->hd[1] = hd[1];
    p->in = in;
    p->out = out;
    return p;
}

fftw_plan fftw_plan_guru_r2r(int rank, const fftw_iodim*, int howmany_rank, const fftw_iodim* howmany_dims, double* in,
                             double* out, const fftw_r2r_kind*, unsigned) {
    return guru_copy(rank, howmany_rank, howmany_dims, in, out, K_COPY);
}

fftw_plan fftw_plan_guru_dft(int rank, const fftw_iodim*, int howmany_rank, const fftw_iodim* howmany_dims, fftw_complex* in,
                             fftw_complex* out, int, unsigned) {
    return guru_copy(rank, howmany_rank, howmany_dims, in, out, K_COPYC);
}

static void exec_any(const fftw_plan p, void* in, void* out) {
    switch (p->kind) {
        case K_DFT: exec_dft(p, (const double*)in, (double*)out); break;
        case K_R2C: exec_r2c(p, (const double*)in, (double*)out); break;
        case K_C2R: exec_c2r(p, (const double*)in, (double*)out); break;
        case K_R2R: exec_r2r(p, (const double*)in, (double*)out); break;
        case K_COPY: exec_copy(p, (const double*)in, (double*)out, 1); break;
        case K_COPYC: exec_copy(p, (const double*)in, (double*)out, 2); break;
    }
}

void fftw_execute(const fftw_plan p) { exec_any(p, p->in, p->out); }
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) { exec_any(p, in, out); }
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) { exec_any(p, in, out); }
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) { exec_any(p, in, out); }
void fftw_execute_r2r(const fftw_plan p, double* in, double* out) { exec_any(p, in, out); }
void fftw_destroy_plan(fftw_plan p) { delete p; }

// no SIMD alignment requirement: any double-aligned pointer is aligned
int fftw_alignment_of(double* p) { return (int)((uintptr_t)p % sizeof(double)); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}
int fftw_import_wisdom_from_filename(const char*) { return 0; }
int fftw_export_wisdom_to_filename(const char*) { return 0; }

}  // extern "C"
