/*
 * mkl.h -- a small stand-in for the parts of Intel MKL that the reference's
 * FGMRES path calls, so that the reference's own C++ sources compile and run
 * here with g++ (the oracle's "_ref" build; test infrastructure only).
 *
 * Only the routines on the FGMRES / BCGSTAB path are implemented
 * (oracle/mkl_standin/mkl_standin.cpp): PARDISO phases 11/22/33/-1 for
 * complex unsymmetric CSR (mtype 13) as a banded LU with partial pivoting,
 * the strided complex 1D DFTI transform as a direct DFT, and the BLAS/LAPACK
 * calls zdotc, zaxpy, dznrm2, zcopy, zdscal, zscal, zgemv, zgels, zlange,
 * dlange and mkl_zcsrgemv, each following the routine's published
 * definition.  Every other MKL routine the reference mentions is declared
 * here with a C variadic prototype and aborts with a message if called.
 *
 * The reference includes this header after `#define MKL_Complex16 dtype`
 * (std::complex<double>), so the prototypes below use MKL_Complex16.
 */
#pragma once
#include <stddef.h>

#define MKL_INT int
#define MKL_LONG long

#ifndef MKL_Complex16
#include <complex>
#define MKL_Complex16 std::complex<double>
#endif
#ifndef MKL_Complex8
#include <complex>
#define MKL_Complex8 std::complex<float>
#endif

typedef void *_MKL_DSS_HANDLE_t;

/* ---- implemented -------------------------------------------------------- */
extern "C" {
void pardisoinit(_MKL_DSS_HANDLE_t pt, const MKL_INT *mtype, MKL_INT *iparm);
void pardiso(_MKL_DSS_HANDLE_t pt, const MKL_INT *maxfct, const MKL_INT *mnum, const MKL_INT *mtype,
             const MKL_INT *phase, const MKL_INT *n, const void *a, const MKL_INT *ia, const MKL_INT *ja,
             MKL_INT *perm, const MKL_INT *nrhs, MKL_INT *iparm, const MKL_INT *msglvl, void *b, void *x,
             MKL_INT *error);
void mkl_set_num_threads(int n);
}

void zdotc(MKL_Complex16 *pres, const MKL_INT *n, const MKL_Complex16 *x, const MKL_INT *incx,
           const MKL_Complex16 *y, const MKL_INT *incy);
void zaxpy(const MKL_INT *n, const MKL_Complex16 *alpha, const MKL_Complex16 *x, const MKL_INT *incx,
           MKL_Complex16 *y, const MKL_INT *incy);
double dznrm2(const MKL_INT *n, const MKL_Complex16 *x, const MKL_INT *incx);
void zcopy(const MKL_INT *n, const MKL_Complex16 *x, const MKL_INT *incx, MKL_Complex16 *y, const MKL_INT *incy);
void zdscal(const MKL_INT *n, const double *a, MKL_Complex16 *x, const MKL_INT *incx);
void zscal(const MKL_INT *n, const MKL_Complex16 *a, MKL_Complex16 *x, const MKL_INT *incx);
void zgemv(const char *trans, const MKL_INT *m, const MKL_INT *n, const MKL_Complex16 *alpha,
           const MKL_Complex16 *a, const MKL_INT *lda, const MKL_Complex16 *x, const MKL_INT *incx,
           const MKL_Complex16 *beta, MKL_Complex16 *y, const MKL_INT *incy);
void zgels(const char *trans, const MKL_INT *m, const MKL_INT *n, const MKL_INT *nrhs, MKL_Complex16 *a,
           const MKL_INT *lda, MKL_Complex16 *b, const MKL_INT *ldb, MKL_Complex16 *work,
           const MKL_INT *lwork, MKL_INT *info);
double zlange(const char *norm, const MKL_INT *m, const MKL_INT *n, const MKL_Complex16 *a,
              const MKL_INT *lda, double *work);
double dlange(const char *norm, const MKL_INT *m, const MKL_INT *n, const double *a, const MKL_INT *lda,
              double *work);
float clange(const char *norm, const MKL_INT *m, const MKL_INT *n, const MKL_Complex8 *a, const MKL_INT *lda,
             float *work);
void zlacpy(const char *uplo, const MKL_INT *m, const MKL_INT *n, const MKL_Complex16 *a, const MKL_INT *lda,
            MKL_Complex16 *b, const MKL_INT *ldb);
void dlacpy(const char *uplo, const MKL_INT *m, const MKL_INT *n, const double *a, const MKL_INT *lda,
            double *b, const MKL_INT *ldb);
void mkl_zcsrgemv(const char *transa, const MKL_INT *m, const MKL_Complex16 *a, const MKL_INT *ia,
                  const MKL_INT *ja, const MKL_Complex16 *x, MKL_Complex16 *y);

/* sparse matrix checker: accepted and reported as consistent */
typedef enum { MKL_ZERO_BASED = 0, MKL_ONE_BASED = 1 } sparse_matrix_indexing;
typedef enum { MKL_GENERAL_STRUCTURE = 0, MKL_UPPER_TRIANGULAR = 1, MKL_LOWER_TRIANGULAR = 2,
               MKL_STRUCTURAL_SYMMETRIC = 3 } sparse_matrix_structures;
typedef enum { MKL_CSR = 0 } sparse_matrix_formats;
typedef enum { MKL_NO_PRINT = 0, MKL_PRINT = 1 } sparse_matrix_message_levels;
typedef enum { MKL_C_STYLE = 0, MKL_FORTRAN_STYLE = 1 } sparse_matrix_print_styles;
typedef struct _sparse_struct {
    MKL_INT n;
    MKL_INT *csr_ia;
    MKL_INT *csr_ja;
    MKL_INT check_result[3];
    sparse_matrix_indexing indexing;
    sparse_matrix_structures matrix_structure;
    sparse_matrix_formats matrix_format;
    sparse_matrix_message_levels message_level;
    sparse_matrix_print_styles print_style;
} sparse_struct;
void sparse_matrix_checker_init(sparse_struct *handle);
int sparse_matrix_checker(sparse_struct *handle);

/* ---- declared only: abort if reached ------------------------------------ */
extern "C" {
void zgemm(...); void ztrsm(...); void zgetrf(...); void zlaswp(...);
void mkl_zomatadd(...); void zsyrk(...); void zsymm(...); void zpotrf(...); void mkl_zimatcopy(...);
void zgetri(...); void mkl_zomatcopy(...); void zgesvd(...); void zaxpby(...); void zgetrs(...);
void zgecon(...); void dgemm(...); void dgemv(...); void dsymv(...); void dsymm(...);
void daxpby(...); void dgesvd(...); void mkl_dimatcopy(...); void mkl_domatcopy(...); void mkl_domatadd(...);
void mkl_dcsrgemv(...); void mkl_zdnscsr(...); void dsyrk(...); void dpotrf(...); void dtrsm(...);
void dgetrf(...); void dgetri(...); void dlaswp(...); void dscal(...); void daxpy(...); void dcopy(...);
double ddot(...); double dnrm2(...); void dgeqrf(...); void zgeqrf(...); void dgels(...); void zlaset(...);
void dlaset(...); void zungqr(...); void dorgqr(...); void zgesv(...); void dgesv(...); void zhemm(...);
void ztrmm(...); void dtrmm(...);
}
