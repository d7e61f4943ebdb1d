/*
 * Forwards the reference's LAPACK/BLAS calls to the LAPACK bundled with scipy
 * (symbols scipy_<name>_, 32-bit integers, Fortran calling convention with
 * hidden string lengths).  Test infrastructure only.
 */
#include "mkl.h"

#include <stddef.h>

typedef size_t flen;

void scipy_dgeqrf_(const int*, const int*, double*, const int*, double*, double*, const int*,
                   int*);
void scipy_dormqr_(const char*, const char*, const int*, const int*, const int*, const double*,
                   const int*, const double*, double*, const int*, double*, const int*, int*,
                   flen, flen);
void scipy_dtrtrs_(const char*, const char*, const char*, const int*, const int*,
                   const double*, const int*, double*, const int*, int*, flen, flen, flen);
void scipy_dgemv_(const char*, const int*, const int*, const double*, const double*,
                  const int*, const double*, const int*, const double*, double*, const int*,
                  flen);
void scipy_dgemm_(const char*, const char*, const int*, const int*, const int*, const double*,
                  const double*, const int*, const double*, const int*, const double*, double*,
                  const int*, flen, flen);
void scipy_dlarf_(const char*, const int*, const int*, const double*, const int*,
                  const double*, double*, const int*, double*, flen);
void scipy_dgetrf_(const int*, const int*, double*, const int*, int*, int*);
void scipy_dgetri_(const int*, double*, const int*, const int*, double*, const int*, int*);

void dgeqrf(const int* m, const int* n, double* a, const int* lda, double* tau, double* work,
            const int* lwork, int* info)
{
    scipy_dgeqrf_(m, n, a, lda, tau, work, lwork, info);
}
void dgeqrf_(const int* m, const int* n, double* a, const int* lda, double* tau, double* work,
             const int* lwork, int* info)
{
    scipy_dgeqrf_(m, n, a, lda, tau, work, lwork, info);
}
void dormqr(const char* side, const char* trans, const int* m, const int* n, const int* k,
            const double* a, const int* lda, const double* tau, double* c, const int* ldc,
            double* work, const int* lwork, int* info)
{
    scipy_dormqr_(side, trans, m, n, k, a, lda, tau, c, ldc, work, lwork, info, 1, 1);
}
void dormqr_(const char* side, const char* trans, const int* m, const int* n, const int* k,
             const double* a, const int* lda, const double* tau, double* c, const int* ldc,
             double* work, const int* lwork, int* info)
{
    scipy_dormqr_(side, trans, m, n, k, a, lda, tau, c, ldc, work, lwork, info, 1, 1);
}
void dtrtrs(const char* uplo, const char* trans, const char* diag, const int* n,
            const int* nrhs, const double* a, const int* lda, double* b, const int* ldb,
            int* info)
{
    scipy_dtrtrs_(uplo, trans, diag, n, nrhs, a, lda, b, ldb, info, 1, 1, 1);
}
void dtrtrs_(const char* uplo, const char* trans, const char* diag, const int* n,
             const int* nrhs, const double* a, const int* lda, double* b, const int* ldb,
             int* info)
{
    scipy_dtrtrs_(uplo, trans, diag, n, nrhs, a, lda, b, ldb, info, 1, 1, 1);
}
void dgemv(const char* trans, const int* m, const int* n, const double* alpha,
           const double* a, const int* lda, const double* x, const int* incx,
           const double* beta, double* y, const int* incy)
{
    scipy_dgemv_(trans, m, n, alpha, a, lda, x, incx, beta, y, incy, 1);
}
void dgemm(const char* transa, const char* transb, const int* m, const int* n, const int* k,
           const double* alpha, const double* a, const int* lda, const double* b,
           const int* ldb, const double* beta, double* c, const int* ldc)
{
    scipy_dgemm_(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, 1, 1);
}
void dlarf_(const char* side, const int* m, const int* n, const double* v, const int* incv,
            const double* tau, double* c, const int* ldc, double* work)
{
    scipy_dlarf_(side, m, n, v, incv, tau, c, ldc, work, 1);
}
void dgetrf_(const int* m, const int* n, double* a, const int* lda, int* ipiv, int* info)
{
    scipy_dgetrf_(m, n, a, lda, ipiv, info);
}
void dgetri_(const int* n, double* a, const int* lda, const int* ipiv, double* work,
             const int* lwork, int* info)
{
    scipy_dgetri_(n, a, lda, ipiv, work, lwork, info);
}
