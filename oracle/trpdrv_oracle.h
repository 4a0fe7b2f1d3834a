/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the reference CCSD(T) triples body, used as the checker for the
 * product library (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg only).
 * Nothing in the product links or calls this.  Parity of this restatement is pinned against the
 * reference itself, compiled unmodified from its sources by oracle/Makefile into oracle/_ref/
 * (tests/test_oracle.py), and against the reference driver's known-answer print.
 *
 * Follows:
 *   omp/ccsd_trpdrv_omp_cbody.c:31-145  (16 DGEMMs, eaijk, tengy call, i!=k gated accumulation)
 *   omp/ccsd_tengy_c99.c:5-119          (tengy (b,c) reduction, outputs overwritten)
 *   omp/test.c:160-195                  (klo / j / i / k loop bounds of the driver)
 */
#ifndef TRPDRV_ORACLE_H
#define TRPDRV_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One synthetic system laid out so every pointer the reference body takes is a slice:
 *   t2  [nocc j][nocc x][nvir][nvir]   tij = t2[j][i],  tkj = t2[j][k]
 *   jvv [nocc x][nvir][nvir]           jia = jvv[i],    jka = jvv[k]      (kvv likewise)
 *   tov [nocc x][nvir*nocc]            tia = tov[i],    tka = tov[k]      (xov likewise)
 *   jov [nocc j][nocc x][nocc*nvir]    jij = jov[j][i], jkj = jov[j][k]   (kov likewise)
 *   dintc, dintx, t1v [nocc x][nvir]   *1 = [i], *2 = [k]
 *   eorb [ncor+nocc+nvir]; a = 1-based orbital index of the fixed virtual. */
typedef struct oracle_system {
    int ncor, nocc, nvir, a;
    const double *eorb, *t2, *jvv, *kvv, *tov, *xov, *jov, *kov, *dintc, *dintx, *t1v;
} oracle_system;

/* Column-major C = alpha*op(A)*op(B) + beta*C with a plain triple loop (the call sites are
 * omp/ccsd_trpdrv_omp_cbody.c:71-116; ta/tb are 'N' or 'T'). */
void oracle_dgemm(char ta, char tb, int m, int n, int k, double alpha,
                  const double *A, int lda, const double *B, int ldb,
                  double beta, double *C, int ldc);

/* Same argument list and meaning as ccsd_tengy_omp (omp/ccsd_tengy_c99.c:5-14). */
void oracle_tengy(const double *f1n, const double *f1t, const double *f2n, const double *f2t,
                  const double *f3n, const double *f3t, const double *f4n, const double *f4t,
                  const double *dintc1, const double *dintx1, const double *t1v1,
                  const double *dintc2, const double *dintx2, const double *t1v2,
                  const double *eorb, double eaijk,
                  double *emp4i, double *emp5i, double *emp4k, double *emp5k,
                  int ncor, int nocc, int nvir);

/* Same argument list and meaning as ccsd_trpdrv_omp_cbody_ (omp/ccsd_trpdrv_omp_cbody.c:31-44). */
void oracle_cbody(double *f1n, double *f1t, double *f2n, double *f2t,
                  double *f3n, double *f3t, double *f4n, double *f4t, double *eorb,
                  int *ncor, int *nocc, int *nvir, double *emp4, double *emp5,
                  int *a, int *i, int *j, int *k, int *klo,
                  double *tij, double *tkj, double *tia, double *tka, double *xia, double *xka,
                  double *jia, double *jka, double *kia, double *kka,
                  double *jij, double *jkj, double *kij, double *kkj,
                  double *dintc1, double *dintx1, double *t1v1,
                  double *dintc2, double *dintx2, double *t1v2);

/* Number of (i,j,k) triples the reference driver visits for one `a` (nkpass-independent). */
int64_t oracle_count_triples(int nocc);

/* Triples in the driver's order (omp/test.c:160-165), 1-based, 4 ints each: i, j, k, klo. */
int64_t oracle_enumerate(int nocc, int nkpass, int32_t *ijkl);

/* Per-triple body signature shared by the restatement and the compiled reference body. */
typedef void (*oracle_body_fn)(double *, double *, double *, double *, double *, double *,
                               double *, double *, double *, int *, int *, int *, double *,
                               double *, int *, int *, int *, int *, int *, double *, double *,
                               double *, double *, double *, double *, double *, double *,
                               double *, double *, double *, double *, double *, double *,
                               double *, double *, double *, double *, double *, double *);
typedef void (*oracle_tengy_fn)(const double *, const double *, const double *, const double *,
                                const double *, const double *, const double *, const double *,
                                const double *, const double *, const double *, const double *,
                                const double *, const double *, const double *, double,
                                double *, double *, double *, double *, int, int, int);

/* Runs triples [t_begin, t_end) of the driver order through `body` (NULL = oracle_cbody) on the
 * system's slices.  For each triple it records, in out[4*t..], emp4i, emp5i, emp4k, emp5k taken by
 * calling `tengy` (NULL = oracle_tengy) on the f arrays the body left behind, and it checks that
 * the body's own accumulation equals emp4i+[i!=k]emp4k (the return value counts mismatches above
 * 1e-12 relative).  The totals over the range are summed in long double with Neumaier
 * compensation and returned in tot[0] (emp4), tot[1] (emp5).  nthreads <= 0 uses OpenMP's default. */
int64_t oracle_run_system(const oracle_system *s, int nkpass, int64_t t_begin, int64_t t_end,
                          oracle_body_fn body, oracle_tengy_fn tengy, int nthreads,
                          double *out, double *tot);

/* Compensated (long double, Neumaier) total of per-triple records produced above:
 * tot[0] = sum emp4i + [i!=k] emp4k, tot[1] likewise for emp5. */
void oracle_sum_records(const double *rec, const int32_t *ijkl, int64_t n, double *tot);

/* Seeded synthetic inputs, restated from the product generator's published recipe so that the
 * oracle and the reference arm of the benchmark need nothing from the product library.  Tensor ids
 * 0..10 are eorb, t2, jvv, kvv, tov, xov, jov, kov, dintc, dintx, t1v (the slice layout above);
 * dist 0 = uniform, 1 = log-uniform integral magnitudes.  Element e of tensor w under seed s is
 * splitmix64(key(s, w) + e), key(s, w) = splitmix64(s ^ (w + 1) * 0xD1B54A32D192ED03), mapped to
 * [0, 1) by its top 53 bits:
 *   eorb: core -20 + 15u, occupied -2 + 1.5u, virtual 0.2 + 2.8u, each group sorted ascending;
 *   t2 -0.05 + 0.1u; tov, xov, t1v -0.02 + 0.04u; integrals -0.1 + 0.2u, or with dist 1 a magnitude
 *   10^(-6u) with the sign of the hash's lowest bit (set = negative).
 * Returns the element count written, or -1 on bad arguments (n must equal oracle_tensor_elems). */
int64_t oracle_tensor_elems(int tensor, int ncor, int nocc, int nvir);
int64_t oracle_synth_fill(int tensor, int ncor, int nocc, int nvir, uint64_t seed, int dist,
                          double *out, int64_t n);

/* The reference driver's timed loop (omp/test.c:160-195) without any extra work: triples
 * [t_begin, t_end) of the driver order, one serial call of `body` each, emp4/emp5 accumulated by the
 * body itself through its pointers (starting from *emp4, *emp5).  The f scratch is allocated once.
 * This is what the CPU baseline times. */
void oracle_time_body(const oracle_system *s, int nkpass, int64_t t_begin, int64_t t_end,
                      oracle_body_fn body, double *emp4, double *emp5);

#ifdef __cplusplus
}
#endif
#endif
