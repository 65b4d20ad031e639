/*
 * mkl_lapack.h -- header shim used only to compile the reference C library as
 * a CPU oracle (see mkl_cblas.h).  Maps the Fortran LAPACK symbols the
 * reference calls (ha_linalg.c, ha_procrustes.c, ha_searchlight.c) onto the
 * `scipy_`-prefixed LAPACK entry points of scipy's bundled OpenBLAS.
 */
#ifndef HA_ORACLE_SHIM_MKL_LAPACK_H
#define HA_ORACLE_SHIM_MKL_LAPACK_H

#include "mkl_cblas.h"

void scipy_dgesdd_(const char *jobz, const MKL_INT *m, const MKL_INT *n, double *a,
                   const MKL_INT *lda, double *s, double *u, const MKL_INT *ldu,
                   double *vt, const MKL_INT *ldvt, double *work, const MKL_INT *lwork,
                   MKL_INT *iwork, MKL_INT *info);
void scipy_sgesdd_(const char *jobz, const MKL_INT *m, const MKL_INT *n, float *a,
                   const MKL_INT *lda, float *s, float *u, const MKL_INT *ldu,
                   float *vt, const MKL_INT *ldvt, float *work, const MKL_INT *lwork,
                   MKL_INT *iwork, MKL_INT *info);
void scipy_dgesvd_(const char *jobu, const char *jobvt, const MKL_INT *m, const MKL_INT *n,
                   double *a, const MKL_INT *lda, double *s, double *u, const MKL_INT *ldu,
                   double *vt, const MKL_INT *ldvt, double *work, const MKL_INT *lwork,
                   MKL_INT *info);
void scipy_sgesvd_(const char *jobu, const char *jobvt, const MKL_INT *m, const MKL_INT *n,
                   float *a, const MKL_INT *lda, float *s, float *u, const MKL_INT *ldu,
                   float *vt, const MKL_INT *ldvt, float *work, const MKL_INT *lwork,
                   MKL_INT *info);
void scipy_dgetrf_(const MKL_INT *m, const MKL_INT *n, double *a, const MKL_INT *lda,
                   MKL_INT *ipiv, MKL_INT *info);
void scipy_sgetrf_(const MKL_INT *m, const MKL_INT *n, float *a, const MKL_INT *lda,
                   MKL_INT *ipiv, MKL_INT *info);
void scipy_sgetri_(const MKL_INT *n, float *a, const MKL_INT *lda, const MKL_INT *ipiv,
                   float *work, const MKL_INT *lwork, MKL_INT *info);

#define dgesdd_ scipy_dgesdd_
#define sgesdd_ scipy_sgesdd_
#define dgesvd_ scipy_dgesvd_
#define sgesvd_ scipy_sgesvd_
#define dgetrf_ scipy_dgetrf_
#define sgetrf_ scipy_sgetrf_
#define sgetri_ scipy_sgetri_

#endif
