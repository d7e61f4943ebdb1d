/*
 * LAPACK/BLAS prototypes in the two spellings the reference MSPAI sources call
 * (MKL's un-suffixed C names, e.g. Spai_Sub.cpp:93-173, and the Fortran "_"
 * names, e.g. qrupdates.cpp:112-160, Matrix.imp:3021-3028).  Both forward to
 * the LAPACK that scipy ships (lapack_forward.c).  Test infrastructure only.
 */
#ifndef ORACLE_SHIM_MKL_H
#define ORACLE_SHIM_MKL_H

#ifdef __cplusplus
extern "C" {
#endif

void dgeqrf(const int* m, const int* n, double* a, const int* lda, double* tau, double* work,
            const int* lwork, int* info);
void dormqr(const char* side, const char* trans, const int* m, const int* n, const int* k,
            const double* a, const int* lda, const double* tau, double* c, const int* ldc,
            double* work, const int* lwork, int* info);
void dtrtrs(const char* uplo, const char* trans, const char* diag, const int* n,
            const int* nrhs, const double* a, const int* lda, double* b, const int* ldb,
            int* info);
void dgemv(const char* trans, const int* m, const int* n, const double* alpha,
           const double* a, const int* lda, const double* x, const int* incx,
           const double* beta, double* y, const int* incy);
void dgemm(const char* transa, const char* transb, const int* m, const int* n, const int* k,
           const double* alpha, const double* a, const int* lda, const double* b,
           const int* ldb, const double* beta, double* c, const int* ldc);

void dgeqrf_(const int* m, const int* n, double* a, const int* lda, double* tau, double* work,
             const int* lwork, int* info);
void dormqr_(const char* side, const char* trans, const int* m, const int* n, const int* k,
             const double* a, const int* lda, const double* tau, double* c, const int* ldc,
             double* work, const int* lwork, int* info);
void dtrtrs_(const char* uplo, const char* trans, const char* diag, const int* n,
             const int* nrhs, const double* a, const int* lda, double* b, const int* ldb,
             int* info);
void dlarf_(const char* side, const int* m, const int* n, const double* v, const int* incv,
            const double* tau, double* c, const int* ldc, double* work);
void dgetrf_(const int* m, const int* n, double* a, const int* lda, int* ipiv, int* info);
void dgetri_(const int* n, double* a, const int* lda, const int* ipiv, double* work,
             const int* lwork, int* info);

#ifdef __cplusplus
}
#endif

#endif
