/*
 * Test infrastructure only: a minimal stand-in for <mkl.h> so that the
 * unmodified reference sources build against the LP64 OpenBLAS that ships
 * inside this Python environment.  It declares the standard CBLAS / LAPACKE
 * entry points the reference calls (six of them, plus the Fortran zheevd_
 * used by an inline helper in util/general.h) with their published
 * signatures; OpenBLAS exports all of them unprefixed.
 *
 * Nothing in the product links this header.
 */
#ifndef DMRG_ORACLE_SHIM_MKL_H_
#define DMRG_ORACLE_SHIM_MKL_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef int MKL_INT;
typedef int lapack_int;

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb,
                 MKL_INT m, MKL_INT n, MKL_INT k, double alpha, const double* a,
                 MKL_INT lda, const double* b, MKL_INT ldb, double beta, double* c,
                 MKL_INT ldc);
void cblas_zgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb,
                 MKL_INT m, MKL_INT n, MKL_INT k, const void* alpha, const void* a,
                 MKL_INT lda, const void* b, MKL_INT ldb, const void* beta, void* c,
                 MKL_INT ldc);

lapack_int LAPACKE_dgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n,
                          double* a, lapack_int lda, double* s, double* u, lapack_int ldu,
                          double* vt, lapack_int ldvt, double* superb);
lapack_int LAPACKE_zgesdd(int layout, char jobz, lapack_int m, lapack_int n, void* a,
                          lapack_int lda, double* s, void* u, lapack_int ldu, void* vt,
                          lapack_int ldvt);
lapack_int LAPACKE_dsyevd(int layout, char jobz, char uplo, lapack_int n, double* a,
                          lapack_int lda, double* w);
lapack_int LAPACKE_zheevd(int layout, char jobz, char uplo, lapack_int n, void* a,
                          lapack_int lda, double* w);

void zheevd_(const char* jobz, const char* uplo, const int* n, void* a, const int* lda,
             double* w, void* work, const int* lwork, double* rwork, const int* lrwork,
             int* iwork, const int* liwork, int* info);
#define zheevd zheevd_

void openblas_set_num_threads(int num_threads);

#ifdef __cplusplus
}
#endif

#endif
