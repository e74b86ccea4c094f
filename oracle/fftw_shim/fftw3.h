/*
 * Test-oracle infrastructure: never linked into the product library.
 *
 * A project-written stand-in for the subset of the FFTW3 API that the
 * reference's ElectrostaticField.cpp calls (src/placement/ElectrostaticField.cpp:
 * FftwRealArray/FftwComplexArray/FftwPlan wrappers, initializeNeumannPlans,
 * initializePeriodicPlans).  FFTW3 itself is not installed here, so the
 * reference CPU field solver is compiled against this header instead.
 *
 * Semantics follow FFTW's published definitions (unnormalized transforms):
 *   REDFT10 (DCT-II):  Y_k = 2 sum_j X_j cos(pi k (2j+1) / (2N))
 *   REDFT01 (DCT-III): Y_k = X_0 + 2 sum_{j>=1} X_j cos(pi j (2k+1) / (2N))
 *   RODFT01 (DST-III): Y_k = (-1)^k X_{N-1} + 2 sum_{j<N-1} X_j sin(pi (j+1)(2k+1) / (2N))
 *   r2c / c2r 2-D: forward sign -1, backward sign +1, no 1/N scaling.
 */
#ifndef MPGP_ORACLE_FFTW3_SHIM_H
#define MPGP_ORACLE_FFTW3_SHIM_H

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

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_ESTIMATE (1U << 6)

double* fftw_alloc_real(size_t n);
fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);

fftw_plan fftw_plan_r2r_2d(int n0, int n1, double* in, double* out, fftw_r2r_kind kind0,
                           fftw_r2r_kind kind1, unsigned flags);
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);

#ifdef __cplusplus
}
#endif

#endif
