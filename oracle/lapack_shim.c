/* Test-oracle infrastructure. Forwards the three LAPACK/BLAS routines the
 * BD_BOX CPU build calls (dpotrf_ at myblas.c:58-61, dtrmv_ at myblas.c:100-103,
 * dsymv_ at diff_alg/diff_equation.c:152-159) to the OpenBLAS 0.3.x that ships
 * inside SciPy, whose exports carry a "scipy_" prefix. Fortran hidden string
 * lengths are passed as 1. */
#include <stddef.h>

void scipy_dpotrf_(const char*, const int*, double*, const int*, int*, size_t);
void scipy_dtrmv_(const char*, const char*, const char*, const int*, const double*,
                  const int*, double*, const int*, size_t, size_t, size_t);
void scipy_dsymv_(const char*, const int*, const double*, const double*, const int*,
                  const double*, const int*, const double*, double*, const int*, size_t);

void dpotrf_(const char* uplo, const int* n, double* a, const int* lda, int* info)
{
    scipy_dpotrf_(uplo, n, a, lda, info, 1);
}

void dtrmv_(const char* uplo, const char* trans, const char* diag, const int* n,
            const double* a, const int* lda, double* x, const int* incx)
{
    scipy_dtrmv_(uplo, trans, diag, n, a, lda, x, incx, 1, 1, 1);
}

void dsymv_(const char* uplo, const int* n, const double* alpha, const double* a,
            const int* lda, const double* x, const int* incx, const double* beta,
            double* y, const int* incy)
{
    scipy_dsymv_(uplo, n, alpha, a, lda, x, incx, beta, y, incy, 1);
}
