/*
 * trpdrv_fp32.h — C ABI of libtrpdrv_b200_fp32.so, the FP32 parity form of the triples body.
 *
 * The reference's single-precision variant (gpu-omp/) declares the SAME entry-point names as the
 * double-precision one with float arrays, so this form lives in its own library: a program built
 * against the gpu-omp signatures (gpu-omp/test.c:24-62) links against libtrpdrv_b200_fp32.so
 * unchanged.  The 16 GEMMs run in IEEE FP32 on the GPU (no TF32), the energies in float, as the
 * reference's cblas_sgemm calls and float tengy loop do.  It exists to compare with that variant's
 * numbers; the FP64 library is the one to use for energies.
 *
 * Conventions as in trpdrv.h: arguments by reference (Fortran-callable), 1-based orbital indices,
 * column-major matrices, caller-owned HOST buffers; f1n..f4t are scratch, written back only when
 * TRPDRV_WRITE_F=1.  Errors print to stderr and abort, or with TRPDRV_ON_ERROR=return leave the
 * outputs unchanged and set trpdrv_fp32_last_error().
 */
#ifndef TRPDRV_B200_FP32_H
#define TRPDRV_B200_FP32_H

#ifdef __cplusplus
extern "C" {
#endif

/* One triple in FP32.  Replaces the float ccsd_trpdrv_omp_cbody_ of gpu-omp/ccsd_trpdrv_omp_cbody.c:38-51
 * (caller prototype gpu-omp/test.c:39-52). */
void ccsd_trpdrv_omp_cbody_(float *f1n, float *f1t, float *f2n, float *f2t,
                            float *f3n, float *f3t, float *f4n, float *f4t, float *eorb,
                            int *ncor, int *nocc, int *nvir, float *emp4, float *emp5,
                            int *a, int *i, int *j, int *k, int *klo,
                            float *tij, float *tkj, float *tia, float *tka,
                            float *xia, float *xka, float *jia, float *jka,
                            float *kia, float *kka, float *jij, float *jkj,
                            float *kij, float *kkj,
                            float *dintc1, float *dintx1, float *t1v1,
                            float *dintc2, float *dintx2, float *t1v2);

/* Same contract; replaces the float Fortran body that gpu-omp/test.c calls under -DUSE_FORTRAN
 * (gpu-omp/test.c:24-37; gpu-omp/ccsd_trpdrv_omp_f77.f). */
void ccsd_trpdrv_omp_fbody_(float *f1n, float *f1t, float *f2n, float *f2t,
                            float *f3n, float *f3t, float *f4n, float *f4t, float *eorb,
                            int *ncor, int *nocc, int *nvir, float *emp4, float *emp5,
                            int *a, int *i, int *j, int *k, int *klo,
                            float *tij, float *tkj, float *tia, float *tka,
                            float *xia, float *xka, float *jia, float *jka,
                            float *kia, float *kka, float *jij, float *jkj,
                            float *kij, float *kkj,
                            float *dintc1, float *dintx1, float *t1v1,
                            float *dintc2, float *dintx2, float *t1v2);

/* The float (b,c) energy reduction on host f arrays; outputs overwritten.  Replaces the float
 * ccsd_tengy_omp of gpu-omp/ccsd_tengy_c99.c:5-14. */
void ccsd_tengy_omp(const float *f1n, const float *f1t, const float *f2n, const float *f2t,
                    const float *f3n, const float *f3t, const float *f4n, const float *f4t,
                    const float *dintc1, const float *dintx1, const float *t1v1,
                    const float *dintc2, const float *dintx2, const float *t1v2,
                    const float *eorb, const float eaijk,
                    float *emp4i, float *emp5i, float *emp4k, float *emp5k,
                    const int ncor, const int nocc, const int nvir);

/* Status of this thread's last failing call in this library (0 = none; 1 invalid argument, 2 CUDA
 * error, 3 out of memory, 4 no sm_100 device) and its message.  No counterpart in the reference. */
int trpdrv_fp32_last_error(void);
const char *trpdrv_fp32_last_error_message(void);

#ifdef __cplusplus
}
#endif
#endif /* TRPDRV_B200_FP32_H */
