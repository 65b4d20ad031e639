/*
 * mkl_cblas.h -- header shim used only to compile the reference C library as
 * a CPU oracle.  The reference includes <mkl_cblas.h> on Linux
 * (ha_common.h:26-33); this image has no MKL, so the CBLAS names the
 * reference calls are mapped onto the `scipy_`-prefixed CBLAS entry points
 * exported by the OpenBLAS build that ships inside scipy (scipy.libs).
 * Only the routines the reference uses are declared.
 */
#ifndef HA_ORACLE_SHIM_MKL_CBLAS_H
#define HA_ORACLE_SHIM_MKL_CBLAS_H

typedef int MKL_INT; /* LP64 OpenBLAS: 32-bit Fortran integers */

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

void scipy_cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                       MKL_INT m, MKL_INT n, MKL_INT k, double alpha,
                       const double *a, MKL_INT lda, const double *b, MKL_INT ldb,
                       double beta, double *c, MKL_INT ldc);
void scipy_cblas_sgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                       MKL_INT m, MKL_INT n, MKL_INT k, float alpha,
                       const float *a, MKL_INT lda, const float *b, MKL_INT ldb,
                       float beta, float *c, MKL_INT ldc);
void scipy_cblas_dgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, MKL_INT m, MKL_INT n,
                       double alpha, const double *a, MKL_INT lda, const double *x,
                       MKL_INT incx, double beta, double *y, MKL_INT incy);
void scipy_cblas_dger(CBLAS_LAYOUT layout, MKL_INT m, MKL_INT n, double alpha,
                      const double *x, MKL_INT incx, const double *y, MKL_INT incy,
                      double *a, MKL_INT lda);
void scipy_cblas_sger(CBLAS_LAYOUT layout, MKL_INT m, MKL_INT n, float alpha,
                      const float *x, MKL_INT incx, const float *y, MKL_INT incy,
                      float *a, MKL_INT lda);
void scipy_cblas_dscal(MKL_INT n, double alpha, double *x, MKL_INT incx);
void scipy_cblas_sscal(MKL_INT n, float alpha, float *x, MKL_INT incx);

#define cblas_dgemm scipy_cblas_dgemm
#define cblas_sgemm scipy_cblas_sgemm
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_dger  scipy_cblas_dger
#define cblas_sger  scipy_cblas_sger
#define cblas_dscal scipy_cblas_dscal
#define cblas_sscal scipy_cblas_sscal

#endif
