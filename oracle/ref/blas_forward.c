/* BLAS / LAPACK for the reference's CPU path when it is built as a test oracle:
 * each Fortran symbol the reference declares (src/layer_0_core/math/linear_algebra/
 * blas.hpp, lapack.hpp) forwards to the same routine in the OpenBLAS that scipy
 * ships, whose exports carry a "scipy_" prefix.  Test infrastructure only. */
typedef struct { double re, im; } zc;

#define FWD(ret, name, params, args) \
    extern ret scipy_##name params;  \
    ret name params { return scipy_##name args; }

FWD(void, zgemm_, (const char* ta, const char* tb, const int* m, const int* n, const int* k,
                   const zc* alpha, const zc* a, const int* lda, const zc* b, const int* ldb,
                   const zc* beta, zc* c, const int* ldc),
    (ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc))
FWD(void, dgemm_, (const char* ta, const char* tb, const int* m, const int* n, const int* k,
                   const double* alpha, const double* a, const int* lda, const double* b,
                   const int* ldb, const double* beta, double* c, const int* ldc),
    (ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc))
FWD(void, zgemv_, (const char* t, const int* m, const int* n, const zc* alpha, const zc* a,
                   const int* lda, const zc* x, const int* incx, const zc* beta, zc* y,
                   const int* incy),
    (t, m, n, alpha, a, lda, x, incx, beta, y, incy))
FWD(void, dgemv_, (const char* t, const int* m, const int* n, const double* alpha,
                   const double* a, const int* lda, const double* x, const int* incx,
                   const double* beta, double* y, const int* incy),
    (t, m, n, alpha, a, lda, x, incx, beta, y, incy))
FWD(void, zaxpy_, (const int* n, const zc* alpha, const zc* x, const int* incx, zc* y,
                   const int* incy),
    (n, alpha, x, incx, y, incy))
FWD(void, zdscal_, (const int* n, const double* alpha, zc* x, const int* incx),
    (n, alpha, x, incx))
FWD(double, dznrm2_, (const int* n, const zc* x, const int* incx), (n, x, incx))
FWD(void, zpotrf_, (const char* uplo, const int* n, zc* a, const int* lda, int* info),
    (uplo, n, a, lda, info))
FWD(void, dpotrf_, (const char* uplo, const int* n, double* a, const int* lda, int* info),
    (uplo, n, a, lda, info))
FWD(void, ztrsm_, (const char* side, const char* uplo, const char* ta, const char* diag,
                   const int* m, const int* n, const zc* alpha, const zc* a, const int* lda,
                   zc* b, const int* ldb),
    (side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb))
FWD(void, dtrsm_, (const char* side, const char* uplo, const char* ta, const char* diag,
                   const int* m, const int* n, const double* alpha, const double* a,
                   const int* lda, double* b, const int* ldb),
    (side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb))
FWD(void, zhegv_, (const int* itype, const char* jobz, const char* uplo, const int* n, zc* a,
                   const int* lda, zc* b, const int* ldb, double* w, zc* work, const int* lwork,
                   double* rwork, int* info),
    (itype, jobz, uplo, n, a, lda, b, ldb, w, work, lwork, rwork, info))
FWD(void, dsygv_, (const int* itype, const char* jobz, const char* uplo, const int* n,
                   double* a, const int* lda, double* b, const int* ldb, double* w,
                   double* work, const int* lwork, int* info),
    (itype, jobz, uplo, n, a, lda, b, ldb, w, work, lwork, info))
FWD(void, zheev_, (const char* jobz, const char* uplo, const int* n, zc* a, const int* lda,
                   double* w, zc* work, const int* lwork, double* rwork, int* info),
    (jobz, uplo, n, a, lda, w, work, lwork, rwork, info))
