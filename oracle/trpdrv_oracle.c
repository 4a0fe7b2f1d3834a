/*
 * ORACLE — test infrastructure only (see trpdrv_oracle.h).  The product never links this.
 *
 * A restatement, in our own code, of the reference algorithm:
 *   omp/ccsd_trpdrv_omp_cbody.c:31-145, omp/ccsd_tengy_c99.c:5-119, omp/test.c:160-195.
 * The DGEMM is a plain triple loop instead of the reference's third-party BLAS.
 */
#include "trpdrv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_MIN(x, y) ((x) < (y) ? (x) : (y))

/* Column-major DGEMM, BLAS semantics (beta == 0 does not read C).
 * Call sites: omp/ccsd_trpdrv_omp_cbody.c:71-116. */
void oracle_dgemm(char ta, char tb, int m, int n, int k, double alpha,
                  const double *A, int lda, const double *B, int ldb,
                  double beta, double *C, int ldc)
{
    double stackbuf[1024];
    double *acc = (m <= 1024) ? stackbuf : (double *)malloc(sizeof(double) * (size_t)m);
    const int at = (ta == 'T' || ta == 't');
    const int bt = (tb == 'T' || tb == 't');
    for (int j = 0; j < n; ++j) {
        for (int r = 0; r < m; ++r) acc[r] = 0.0;
        for (int l = 0; l < k; ++l) {
            const double b = bt ? B[j + (size_t)l * ldb] : B[l + (size_t)j * ldb];
            if (!at) {
                const double *col = A + (size_t)l * lda;
                for (int r = 0; r < m; ++r) acc[r] += col[r] * b;
            } else {
                for (int r = 0; r < m; ++r) acc[r] += A[l + (size_t)r * lda] * b;
            }
        }
        double *c = C + (size_t)j * ldc;
        if (beta == 0.0) {
            for (int r = 0; r < m; ++r) c[r] = alpha * acc[r];
        } else {
            for (int r = 0; r < m; ++r) c[r] = alpha * acc[r] + beta * c[r];
        }
    }
    if (acc != stackbuf) free(acc);
}

/* omp/ccsd_tengy_c99.c:52-118: the 32x32-tiled (b,c) loop, run serially.  The four outputs are
 * overwritten, not accumulated (:115-118). */
void oracle_tengy(const double *f1n, const double *f1t, const double *f2n, const double *f2t,
                  const double *f3n, const double *f3t, const double *f4n, const double *f4t,
                  const double *dintc1, const double *dintx1, const double *t1v1,
                  const double *dintc2, const double *dintx2, const double *t1v2,
                  const double *eorb, double eaijk,
                  double *emp4i_, double *emp5i_, double *emp4k_, double *emp5k_,
                  int ncor, int nocc, int nvir)
{
    double emp4i = 0.0, emp5i = 0.0, emp4k = 0.0, emp5k = 0.0;
    const int tile = 32;
    for (int bt = 0; bt < nvir; bt += tile) {
        for (int ct = 0; ct < nvir; ct += tile) {
            for (int b = bt; b < ORACLE_MIN(bt + tile, nvir); ++b) {
                for (int c = ct; c < ORACLE_MIN(ct + tile, nvir); ++c) {
                    /* orbital-energy denominator, :65 */
                    const double denom = -1.0 / (eorb[ncor + nocc + b] + eorb[ncor + nocc + c] + eaijk);
                    const int bc = b + c * nvir;
                    const int cb = c + b * nvir;
                    const double n1bc = f1n[bc], t1bc = f1t[bc], n1cb = f1n[cb], t1cb = f1t[cb];
                    const double n2bc = f2n[bc], t2bc = f2t[bc], n2cb = f2n[cb], t2cb = f2t[cb];
                    const double n3bc = f3n[bc], t3bc = f3t[bc], n3cb = f3n[cb], t3cb = f3t[cb];
                    const double n4bc = f4n[bc], t4bc = f4t[bc], n4cb = f4n[cb], t4cb = f4t[cb];

                    /* quadratic emp4 forms, :91-96 */
                    emp4i += denom * (t1bc + n1cb + t2cb + n3bc + n4cb) * (t1bc - t2bc * 2 - t3bc * 2 + t4bc)
                           - denom * (n1bc + t1cb + n2cb + n3cb) * (t1bc * 2 - t2bc - t3bc + t4bc * 2)
                           + denom * 3 * (n1bc * (n1bc + n3cb + t4cb * 2) + n2bc * t2cb + n3bc * t4bc);
                    emp4k += denom * (n1bc + t1cb + n2cb + t3bc + t4cb) * (n1bc - n2bc * 2 - n3bc * 2 + n4bc)
                           - denom * (t1bc + n1cb + t2cb + t3cb) * (n1bc * 2 - n2bc - n3bc + n4bc * 2)
                           + denom * 3 * (t1bc * (t1bc + t3cb + n4cb * 2) + t2bc * n2cb + t3bc * n4bc);

                    /* linear emp5 forms, :98-111 */
                    const double t1v1b = t1v1[b], t1v2b = t1v2[b];
                    const double dx1c = dintx1[c], dx2c = dintx2[c];
                    const double dc1c = dintc1[c], dc2c = dintc2[c];
                    emp5i += denom * t1v1b * dx1c * (t1bc + n2bc + n4cb - (t3bc + n4bc + n2cb + n1bc + t2bc + n3cb) * 2
                                                      + (n3bc + t4bc + n1cb) * 4)
                           + denom * t1v1b * dc1c * (n1bc + n4bc + t1cb - (n2bc + n3bc + t2cb) * 2);
                    emp5k += denom * t1v2b * dx2c * (n1bc + t2bc + t4cb - (n3bc + t4bc + t2cb + t1bc + n2bc + t3cb) * 2
                                                      + (t3bc + n4bc + t1cb) * 4)
                           + denom * t1v2b * dc2c * (t1bc + t4bc + n1cb - (t2bc + t3bc + n2cb) * 2);
                }
            }
        }
    }
    *emp4i_ = emp4i;
    *emp4k_ = emp4k;
    *emp5i_ = emp5i;
    *emp5k_ = emp5k;
}

/* omp/ccsd_trpdrv_omp_cbody.c:31-145. */
void oracle_cbody(double *f1n, double *f1t, double *f2n, double *f2t,
                  double *f3n, double *f3t, double *f4n, double *f4t, double *eorb,
                  int *ncor_, int *nocc_, int *nvir_, double *emp4_, double *emp5_,
                  int *a_, int *i_, int *j_, int *k_, int *klo_,
                  double *tij, double *tkj, double *tia, double *tka, double *xia, double *xka,
                  double *jia, double *jka, double *kia, double *kka,
                  double *jij, double *jkj, double *kij, double *kkj,
                  double *dintc1, double *dintx1, double *t1v1,
                  double *dintc2, double *dintx2, double *t1v2)
{
    const int ncor = *ncor_, nocc = *nocc_, nvir = *nvir_;
    const size_t lnov = (size_t)nocc * nvir;
    const size_t lnvv = (size_t)nvir * nvir;
    const int k = *k_ - 1;      /* 1-based -> 0-based, :62-63 */
    const int klo = *klo_ - 1;
    const size_t vv = (size_t)(k - klo) * lnvv;
    const size_t ov = (size_t)(k - klo) * lnov;
    const int nv = nvir, no = nocc;

    /* n-side: eight GEMMs, :70-93 */
    oracle_dgemm('N', 'T', nv, nv, nv, 1.0, jia, nv, tkj + vv, nv, 0.0, f1n, nv);
    oracle_dgemm('N', 'N', nv, nv, no, -1.0, tia, nv, kkj + ov, no, 1.0, f1n, nv);
    oracle_dgemm('N', 'T', nv, nv, nv, 1.0, kia, nv, tkj + vv, nv, 0.0, f2n, nv);
    oracle_dgemm('N', 'N', nv, nv, no, -1.0, xia, nv, kkj + ov, no, 1.0, f2n, nv);
    oracle_dgemm('N', 'N', nv, nv, nv, 1.0, jia, nv, tkj + vv, nv, 0.0, f3n, nv);
    oracle_dgemm('N', 'N', nv, nv, no, -1.0, tia, nv, jkj + ov, no, 1.0, f3n, nv);
    oracle_dgemm('N', 'N', nv, nv, nv, 1.0, kia, nv, tkj + vv, nv, 0.0, f4n, nv);
    oracle_dgemm('N', 'N', nv, nv, no, -1.0, xia, nv, jkj + ov, no, 1.0, f4n, nv);
    /* t-side: eight GEMMs, :94-117 */
    oracle_dgemm('N', 'T', nv, nv, nv, 1.0, jka + vv, nv, tij, nv, 0.0, f1t, nv);
    oracle_dgemm('N', 'N', nv, nv, no, -1.0, tka + ov, nv, kij, no, 1.0, f1t, nv);
    oracle_dgemm('N', 'T', nv, nv, nv, 1.0, kka + vv, nv, tij, nv, 0.0, f2t, nv);
    oracle_dgemm('N', 'N', nv, nv, no, -1.0, xka + ov, nv, kij, no, 1.0, f2t, nv);
    oracle_dgemm('N', 'N', nv, nv, nv, 1.0, jka + vv, nv, tij, nv, 0.0, f3t, nv);
    oracle_dgemm('N', 'N', nv, nv, no, -1.0, tka + ov, nv, jij, no, 1.0, f3t, nv);
    oracle_dgemm('N', 'N', nv, nv, nv, 1.0, kka + vv, nv, tij, nv, 0.0, f4t, nv);
    oracle_dgemm('N', 'N', nv, nv, no, -1.0, xka + ov, nv, jij, no, 1.0, f4t, nv);

    const int a = *a_ - 1, i = *i_ - 1, j = *j_ - 1;
    const double eaijk = eorb[a] - (eorb[ncor + i] + eorb[ncor + j] + eorb[ncor + k]);   /* :126 */
    double emp4i, emp5i, emp4k, emp5k;
    oracle_tengy(f1n, f1t, f2n, f2t, f3n, f3t, f4n, f4t, dintc1, dintx1, t1v1, dintc2, dintx2, t1v2,
                 eorb, eaijk, &emp4i, &emp5i, &emp4k, &emp5k, ncor, nocc, nvir);
    double emp4 = *emp4_, emp5 = *emp5_;
    emp4 += emp4i;              /* :133-142 */
    emp5 += emp5i;
    if (*i_ != *k_) {
        emp4 += emp4k;
        emp5 += emp5k;
    }
    *emp4_ = emp4;
    *emp5_ = emp5;
}

int64_t oracle_count_triples(int nocc)
{
    return (int64_t)nocc * nocc * (nocc + 1) / 2;
}

/* omp/test.c:97 (kchunk) and :160-165 (loop bounds); `a` is fixed by the caller. */
int64_t oracle_enumerate(int nocc, int nkpass, int32_t *ijkl)
{
    if (nkpass < 1) nkpass = 1;
    const int kchunk = (nocc - 1) / nkpass + 1;
    int64_t t = 0;
    for (int klo = 1; klo <= nocc; klo += kchunk) {
        const int khi = ORACLE_MIN(nocc, klo + kchunk - 1);
        for (int j = 1; j <= nocc; ++j)
            for (int i = 1; i <= nocc; ++i)
                for (int k = klo; k <= ORACLE_MIN(khi, i); ++k) {
                    if (ijkl) {
                        ijkl[4 * t + 0] = i;
                        ijkl[4 * t + 1] = j;
                        ijkl[4 * t + 2] = k;
                        ijkl[4 * t + 3] = klo;
                    }
                    ++t;
                }
    }
    return t;
}

static void neumaier_add(long double *sum, long double *comp, long double x)
{
    const long double t = *sum + x;
    if (fabsl(*sum) >= fabsl(x))
        *comp += (*sum - t) + x;
    else
        *comp += (x - t) + *sum;
    *sum = t;
}

void oracle_sum_records(const double *rec, const int32_t *ijkl, int64_t n, double *tot)
{
    long double s4 = 0, c4 = 0, s5 = 0, c5 = 0;
    for (int64_t t = 0; t < n; ++t) {
        neumaier_add(&s4, &c4, rec[4 * t + 0]);
        neumaier_add(&s5, &c5, rec[4 * t + 1]);
        if (ijkl[4 * t + 0] != ijkl[4 * t + 2]) {
            neumaier_add(&s4, &c4, rec[4 * t + 2]);
            neumaier_add(&s5, &c5, rec[4 * t + 3]);
        }
    }
    tot[0] = (double)(s4 + c4);
    tot[1] = (double)(s5 + c5);
}

int64_t oracle_run_system(const oracle_system *s, int nkpass, int64_t t_begin, int64_t t_end,
                          oracle_body_fn body, oracle_tengy_fn tengy, int nthreads,
                          double *out, double *tot)
{
    const int nocc = s->nocc, nvir = s->nvir;
    const int64_t ntot = oracle_count_triples(nocc);
    if (t_begin < 0) t_begin = 0;
    if (t_end > ntot) t_end = ntot;
    if (t_end <= t_begin) {
        if (tot) tot[0] = tot[1] = 0.0;
        return 0;
    }
    int32_t *ijkl = (int32_t *)malloc(sizeof(int32_t) * 4 * (size_t)ntot);
    oracle_enumerate(nocc, nkpass, ijkl);
    if (!body) body = (oracle_body_fn)oracle_cbody;
    if (!tengy) tengy = (oracle_tengy_fn)oracle_tengy;
    const size_t lnvv = (size_t)nvir * nvir, lnov = (size_t)nocc * nvir;
    const int64_t n = t_end - t_begin;
    double *rec = out ? out : (double *)malloc(sizeof(double) * 4 * (size_t)n);
    int64_t mismatches = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif

#pragma omp parallel num_threads(nthreads) if (nthreads > 1) reduction(+ : mismatches)
    {
        double *f = (double *)malloc(sizeof(double) * 8 * lnvv);
        double *const f1n = f, *const f1t = f + lnvv, *const f2n = f + 2 * lnvv, *const f2t = f + 3 * lnvv;
        double *const f3n = f + 4 * lnvv, *const f3t = f + 5 * lnvv, *const f4n = f + 6 * lnvv, *const f4t = f + 7 * lnvv;
#pragma omp for schedule(dynamic, 1)
        for (int64_t t = t_begin; t < t_end; ++t) {
            int i = ijkl[4 * t], j = ijkl[4 * t + 1], k = ijkl[4 * t + 2], klo = ijkl[4 * t + 3];
            int ncor = s->ncor, no = nocc, nv = nvir, a = s->a;
            const size_t jb = (size_t)(j - 1) * nocc;
            double *tij = (double *)s->t2 + (jb + (i - 1)) * lnvv;
            double *tkj = (double *)s->t2 + (jb + (klo - 1)) * lnvv;
            double *jia = (double *)s->jvv + (size_t)(i - 1) * lnvv, *jka = (double *)s->jvv + (size_t)(klo - 1) * lnvv;
            double *kia = (double *)s->kvv + (size_t)(i - 1) * lnvv, *kka = (double *)s->kvv + (size_t)(klo - 1) * lnvv;
            double *tia = (double *)s->tov + (size_t)(i - 1) * lnov, *tka = (double *)s->tov + (size_t)(klo - 1) * lnov;
            double *xia = (double *)s->xov + (size_t)(i - 1) * lnov, *xka = (double *)s->xov + (size_t)(klo - 1) * lnov;
            double *jij = (double *)s->jov + (jb + (i - 1)) * lnov, *jkj = (double *)s->jov + (jb + (klo - 1)) * lnov;
            double *kij = (double *)s->kov + (jb + (i - 1)) * lnov, *kkj = (double *)s->kov + (jb + (klo - 1)) * lnov;
            double *dc1 = (double *)s->dintc + (size_t)(i - 1) * nvir, *dc2 = (double *)s->dintc + (size_t)(k - 1) * nvir;
            double *dx1 = (double *)s->dintx + (size_t)(i - 1) * nvir, *dx2 = (double *)s->dintx + (size_t)(k - 1) * nvir;
            double *tv1 = (double *)s->t1v + (size_t)(i - 1) * nvir, *tv2 = (double *)s->t1v + (size_t)(k - 1) * nvir;
            double e4 = 0.0, e5 = 0.0;
            body(f1n, f1t, f2n, f2t, f3n, f3t, f4n, f4t, (double *)s->eorb, &ncor, &no, &nv, &e4, &e5,
                 &a, &i, &j, &k, &klo, tij, tkj, tia, tka, xia, xka, jia, jka, kia, kka, jij, jkj, kij, kkj,
                 dc1, dx1, tv1, dc2, dx2, tv2);
            const double eaijk = s->eorb[a - 1] - (s->eorb[ncor + i - 1] + s->eorb[ncor + j - 1] + s->eorb[ncor + k - 1]);
            double r4i, r5i, r4k, r5k;
            tengy(f1n, f1t, f2n, f2t, f3n, f3t, f4n, f4t, dc1, dx1, tv1, dc2, dx2, tv2, s->eorb, eaijk,
                  &r4i, &r5i, &r4k, &r5k, ncor, nocc, nvir);
            double *o = rec + 4 * (t - t_begin);
            o[0] = r4i;
            o[1] = r5i;
            o[2] = r4k;
            o[3] = r5k;
            double c4 = 0.0 + r4i, c5 = 0.0 + r5i;
            if (i != k) {
                c4 += r4k;
                c5 += r5k;
            }
            const double s4 = fabs(e4) + fabs(c4) + 1e-300, s5 = fabs(e5) + fabs(c5) + 1e-300;
            if (fabs(e4 - c4) > 1e-12 * s4 || fabs(e5 - c5) > 1e-12 * s5) mismatches += 1;
        }
        free(f);
    }
    if (tot) oracle_sum_records(rec, ijkl + 4 * t_begin, n, tot);
    if (rec != out) free(rec);
    free(ijkl);
    return mismatches;
}

/* ---- seeded synthetic inputs (SplitMix64 counter stream; Steele, Lea & Flood, OOPSLA 2014) ---- */

static uint64_t sm64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static int cmp_dbl(const void *p, const void *q)
{
    const double x = *(const double *)p, y = *(const double *)q;
    return (x > y) - (x < y);
}

int64_t oracle_tensor_elems(int tensor, int ncor, int nocc, int nvir)
{
    const int64_t o = nocc > 0 ? nocc : 0, v = nvir > 0 ? nvir : 0;
    switch (tensor) {
    case 0: return (int64_t)(ncor > 0 ? ncor : 0) + o + v; /* eorb */
    case 1: return o * o * v * v;                          /* t2 [j][x][v][v] */
    case 2: case 3: return o * v * v;                      /* jvv, kvv */
    case 4: case 5: return o * v * o;                      /* tov, xov */
    case 6: case 7: return o * o * o * v;                  /* jov, kov */
    case 8: case 9: case 10: return o * v;                 /* dintc, dintx, t1v */
    default: return -1;
    }
}

int64_t oracle_synth_fill(int tensor, int ncor, int nocc, int nvir, uint64_t seed, int dist,
                          double *out, int64_t n)
{
    if (tensor < 0 || tensor > 10 || !out || ncor < 0 || nocc < 1 || nvir < 1 || (dist != 0 && dist != 1))
        return -1;
    if (n != oracle_tensor_elems(tensor, ncor, nocc, nvir)) return -1;
    const uint64_t key = sm64(seed ^ ((uint64_t)(tensor + 1) * 0xD1B54A32D192ED03ull));
    if (tensor == 0) {
        for (int64_t e = 0; e < n; ++e) {
            const double u = (double)(sm64(key + (uint64_t)e) >> 11) * 0x1.0p-53;
            out[e] = e < ncor ? -20.0 + 15.0 * u : (e < ncor + nocc ? -2.0 + 1.5 * u : 0.2 + 2.8 * u);
        }
        qsort(out, (size_t)ncor, sizeof(double), cmp_dbl);
        qsort(out + ncor, (size_t)nocc, sizeof(double), cmp_dbl);
        qsort(out + ncor + nocc, (size_t)nvir, sizeof(double), cmp_dbl);
        return n;
    }
    const double half = tensor == 1 ? 0.05 : ((tensor == 4 || tensor == 5 || tensor == 10) ? 0.02 : 0.1);
    const int integral = !(tensor == 1 || tensor == 4 || tensor == 5 || tensor == 10);
    const int logmag = integral && dist == 1;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n; ++e) {
        const uint64_t h = sm64(key + (uint64_t)e);
        const double u = (double)(h >> 11) * 0x1.0p-53;
        if (logmag) {
            const double m = pow(10.0, -6.0 * u);
            out[e] = (h & 1u) ? -m : m;
        } else {
            out[e] = -half + 2.0 * half * u;
        }
    }
    return n;
}

/* ---- the reference driver's timed loop (omp/test.c:160-195), body calls only ---- */

void oracle_time_body(const oracle_system *s, int nkpass, int64_t t_begin, int64_t t_end,
                      oracle_body_fn body, double *emp4, double *emp5)
{
    const int nocc = s->nocc, nvir = s->nvir;
    const int64_t ntot = oracle_count_triples(nocc);
    if (t_begin < 0) t_begin = 0;
    if (t_end > ntot) t_end = ntot;
    if (t_end <= t_begin || !body) return;
    int32_t *ijkl = (int32_t *)malloc(sizeof(int32_t) * 4 * (size_t)ntot);
    oracle_enumerate(nocc, nkpass, ijkl);
    const size_t lnvv = (size_t)nvir * nvir, lnov = (size_t)nocc * nvir;
    double *f = (double *)malloc(sizeof(double) * 8 * lnvv);
    double e4 = *emp4, e5 = *emp5;
    for (int64_t t = t_begin; t < t_end; ++t) {
        int i = ijkl[4 * t], j = ijkl[4 * t + 1], k = ijkl[4 * t + 2], klo = ijkl[4 * t + 3];
        int ncor = s->ncor, no = nocc, nv = nvir, a = s->a;
        const size_t jb = (size_t)(j - 1) * nocc;
        body(f, f + lnvv, f + 2 * lnvv, f + 3 * lnvv, f + 4 * lnvv, f + 5 * lnvv, f + 6 * lnvv, f + 7 * lnvv,
             (double *)s->eorb, &ncor, &no, &nv, &e4, &e5, &a, &i, &j, &k, &klo,
             (double *)s->t2 + (jb + (i - 1)) * lnvv, (double *)s->t2 + (jb + (klo - 1)) * lnvv,
             (double *)s->tov + (size_t)(i - 1) * lnov, (double *)s->tov + (size_t)(klo - 1) * lnov,
             (double *)s->xov + (size_t)(i - 1) * lnov, (double *)s->xov + (size_t)(klo - 1) * lnov,
             (double *)s->jvv + (size_t)(i - 1) * lnvv, (double *)s->jvv + (size_t)(klo - 1) * lnvv,
             (double *)s->kvv + (size_t)(i - 1) * lnvv, (double *)s->kvv + (size_t)(klo - 1) * lnvv,
             (double *)s->jov + (jb + (i - 1)) * lnov, (double *)s->jov + (jb + (klo - 1)) * lnov,
             (double *)s->kov + (jb + (i - 1)) * lnov, (double *)s->kov + (jb + (klo - 1)) * lnov,
             (double *)s->dintc + (size_t)(i - 1) * nvir, (double *)s->dintx + (size_t)(i - 1) * nvir,
             (double *)s->t1v + (size_t)(i - 1) * nvir, (double *)s->dintc + (size_t)(k - 1) * nvir,
             (double *)s->dintx + (size_t)(k - 1) * nvir, (double *)s->t1v + (size_t)(k - 1) * nvir);
    }
    *emp4 = e4;
    *emp5 = e5;
    free(f);
    free(ijkl);
}
