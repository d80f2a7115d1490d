// FFTW-API subset for compiling the reference's solver sources (src/*.cpp)
// without FFTW: exactly the declarations those sources use (FFTW 3.3
// names, types and constants; the arithmetic behind them is this
// directory's own FP64 FFT, oracle/ref_build/fft_shim.cpp).  Test
// infrastructure of the oracle only.
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;

typedef enum {
    FFTW_R2HC = 0,
    FFTW_HC2R = 1,
    FFTW_DHT = 2,
    FFTW_REDFT00 = 3,
    FFTW_REDFT01 = 4,
    FFTW_REDFT10 = 5,
    FFTW_REDFT11 = 6,
    FFTW_RODFT00 = 7,
    FFTW_RODFT01 = 8,
    FFTW_RODFT10 = 9,
    FFTW_RODFT11 = 10
} fftw_r2r_kind;

typedef struct {
    int n, is, os;
} fftw_iodim;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex* in, double* out, unsigned flags);
fftw_plan fftw_plan_r2r_1d(int n, double* in, double* out, fftw_r2r_kind kind, unsigned flags);
fftw_plan fftw_plan_many_r2r(int rank, const int* n, int howmany, double* in, const int* inembed, int istride, int idist,
                             double* out, const int* onembed, int ostride, int odist, const fftw_r2r_kind* kind,
                             unsigned flags);
fftw_plan fftw_plan_guru_r2r(int rank, const fftw_iodim* dims, int howmany_rank, const fftw_iodim* howmany_dims, double* in,
                             double* out, const fftw_r2r_kind* kind, unsigned flags);
fftw_plan fftw_plan_guru_dft(int rank, const fftw_iodim* dims, int howmany_rank, const fftw_iodim* howmany_dims,
                             fftw_complex* in, fftw_complex* out, int sign, unsigned flags);

void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_execute_r2r(const fftw_plan p, double* in, double* out);
void fftw_destroy_plan(fftw_plan p);

int fftw_alignment_of(double* p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);
int fftw_import_wisdom_from_filename(const char* filename);
int fftw_export_wisdom_to_filename(const char* filename);

#ifdef __cplusplus
}
#endif
