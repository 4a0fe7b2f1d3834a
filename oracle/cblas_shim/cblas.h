/*
 * Minimal CBLAS declaration used ONLY to compile the reference's unmodified
 * omp/ccsd_trpdrv_omp_cbody.c (which does `#include <cblas.h>` when neither
 * MKL nor ACCELERATE is defined, omp/ccsd_trpdrv_omp_cbody.c:14-16), and of its single-precision
 * twin gpu-omp/ccsd_trpdrv_omp_cbody.c (cblas_sgemm), against
 * the OpenBLAS 0.3.30 build that ships inside scipy (scipy.libs/
 * libscipy_openblas-*.so).  That build prefixes its symbols with `scipy_`,
 * so cblas_dgemm / cblas_sgemm are mapped onto scipy_cblas_dgemm / scipy_cblas_sgemm.  The enumerator values are
 * the ones fixed by the CBLAS standard.  32-bit integers (LP64 OpenBLAS).
 *
 * Test infrastructure: this header is part of the oracle build recipe, not
 * of the product library.
 */
#ifndef TRPDRV_ORACLE_CBLAS_SHIM_H
#define TRPDRV_ORACLE_CBLAS_SHIM_H

enum CBLAS_ORDER     { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

void scipy_cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                       int m, int n, int k, double alpha, const double *a, int lda,
                       const double *b, int ldb, double beta, double *c, int ldc);
void scipy_cblas_sgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                       int m, int n, int k, float alpha, const float *a, int lda,
                       const float *b, int ldb, float beta, float *c, int ldc);
void scipy_openblas_set_num_threads(int n);

#define cblas_dgemm scipy_cblas_dgemm
#define cblas_sgemm scipy_cblas_sgemm

#endif
