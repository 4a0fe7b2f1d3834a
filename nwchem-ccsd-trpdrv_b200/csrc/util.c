/*
 * Host-side helpers that need no device: triple enumeration, cost-balanced partitioning and the
 * seeded synthetic input generator.
 */
#include "trpdrv.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int trpdrv_version(void) { return 10100; /* 1.1.0 */ }

int64_t trpdrv_count_triples(int nocc)
{
    if (nocc < 1) return 0;
    return (int64_t)nocc * nocc * (nocc + 1) / 2;
}

/* Loop bounds of the reference driver, omp/test.c:97 (kchunk) and :160-165:
 *   for klo = 1..nocc step kchunk; for j = 1..nocc; for i = 1..nocc; for k = klo..min(khi, i) */
int64_t trpdrv_enumerate_triples(int nocc, int nkpass, int32_t *ijkl)
{
    if (nocc < 1) return 0;
    if (nkpass < 1) nkpass = 1;
    const int kchunk = (nocc - 1) / nkpass + 1;
    int64_t t = 0;
    for (int klo = 1; klo <= nocc; klo += kchunk) {
        const int khi = (nocc < klo + kchunk - 1) ? nocc : klo + kchunk - 1;
        for (int j = 1; j <= nocc; ++j)
            for (int i = 1; i <= nocc; ++i) {
                const int kend = khi < i ? khi : i;
                for (int k = klo; k <= kend; ++k) {
                    if (ijkl) {
                        ijkl[4 * t + 0] = i;
                        ijkl[4 * t + 1] = j;
                        ijkl[4 * t + 2] = k;
                        ijkl[4 * t + 3] = klo;
                    }
                    ++t;
                }
            }
    }
    return t;
}

int trpdrv_partition(const double *cost, int64_t n, int world, int64_t *bounds)
{
    if (world < 1 || n < 0 || !bounds) return TRPDRV_ERR_ARG;
    double total = 0.0;
    for (int64_t t = 0; t < n; ++t) {
        const double c = cost ? cost[t] : 1.0;
        if (!(c >= 0.0)) return TRPDRV_ERR_ARG;
        total += c;
    }
    bounds[0] = 0;
    int64_t t = 0;
    double prefix = 0.0;
    for (int r = 1; r < world; ++r) {
        const double target = total * (double)r / (double)world;
        /* advance while taking the next item keeps the prefix closer to the target */
        while (t < n) {
            const double c = cost ? cost[t] : 1.0;
            if (prefix + 0.5 * c > target) break;
            prefix += c;
            ++t;
        }
        bounds[r] = t;
    }
    bounds[world] = n;
    return TRPDRV_OK;
}

int64_t trpdrv_shard_triples(int nocc, int nkpass, int rank, int world, int32_t *ijk)
{
    if (nocc < 1 || world < 1 || rank < 0 || rank >= world) return -1;
    const int64_t n = trpdrv_count_triples(nocc);
    int32_t *all = (int32_t *)malloc(sizeof(int32_t) * 4 * (size_t)n);
    int64_t *bounds = (int64_t *)malloc(sizeof(int64_t) * (size_t)(world + 1));
    if (!all || !bounds) {
        free(all);
        free(bounds);
        return -1;
    }
    trpdrv_enumerate_triples(nocc, nkpass, all);
    trpdrv_partition(NULL, n, world, bounds);
    const int64_t lo = bounds[rank], hi = bounds[rank + 1];
    if (ijk)
        for (int64_t t = lo; t < hi; ++t) {
            ijk[3 * (t - lo) + 0] = all[4 * t + 0];
            ijk[3 * (t - lo) + 1] = all[4 * t + 1];
            ijk[3 * (t - lo) + 2] = all[4 * t + 2];
        }
    free(all);
    free(bounds);
    return hi - lo;
}

typedef struct order_key {
    int64_t key;
    int32_t idx;
} order_key;

static int order_key_cmp(const void *x, const void *y)
{
    const int64_t a = ((const order_key *)x)->key, b = ((const order_key *)y)->key;
    return (a > b) - (a < b);
}

/* A triple (i, j, k) reads the slices of index i and of index k of T2[j], J, K, JOV[j], KOV[j], TOV
 * and XOV (about 2.5 MB at nvir = 300, nocc = 40).  In the driver order (omp/test.c:160-165) every i
 * sweeps k over 1..i, a cyclic walk over up to nocc slices that an LRU-like L2 cannot hold; here each
 * block of i values stays resident while k streams past it, and consecutive blocks meet at the k
 * slices the previous block touched last. */
int trpdrv_processing_order(const int32_t *ijk, int64_t n, int block, int32_t *order)
{
    if (n < 0 || (n > 0 && (!ijk || !order)) || n > INT32_MAX) return -1;
    if (block <= 0) block = 8;
    order_key *ks = (order_key *)malloc(sizeof(order_key) * (size_t)(n > 0 ? n : 1));
    if (!ks) return -1;
    int64_t run = 0, nblocks = 0;
    while (run < n) {
        int64_t end = run + 1;
        while (end < n && ijk[3 * end + 1] == ijk[3 * run + 1]) ++end;
        int prev_blk = -1;
        for (int64_t t = run; t < end; ++t) {
            const int i = ijk[3 * t] - 1, k = ijk[3 * t + 2] - 1;
            const int blk = i / block;
            if (blk != prev_blk) {
                ++nblocks;
                prev_blk = blk;
            }
            /* the key sorts by block first, so any list (not only the driver's) gives a permutation */
            const int64_t kk = (nblocks & 1) ? (int64_t)(k & 1023) : (int64_t)(1023 - (k & 1023));
            ks[t].key = ((int64_t)(blk & 0xfffff) << 40) | (kk << 20) | (int64_t)(i & 0xfffff);
            ks[t].idx = (int32_t)t;
        }
        qsort(ks + run, (size_t)(end - run), sizeof(order_key), order_key_cmp);
        run = end;
    }
    for (int64_t t = 0; t < n; ++t) order[t] = ks[t].idx;
    free(ks);
    return 0;
}

int64_t trpdrv_upload_spans(const int32_t *ijk, const int32_t *order, int64_t n, int chunks, int64_t *bounds)
{
    if (n < 0 || n > INT32_MAX || chunks < 1 || !bounds || (n > 0 && !ijk)) return -1;
    if (order)
        for (int64_t t = 0; t < n; ++t)
            if (order[t] < 0 || order[t] >= n) return -1;
    int64_t ns = 0, start = 0;
    bounds[0] = 0;
    for (int c = 0; c < chunks && start < n; ++c) {
        int64_t end = c + 1 == chunks ? n : (int64_t)(c + 1) * n / chunks;
        if (end <= start) end = start + 1;
        while (end < n && ijk[3 * (int64_t)(order ? order[end] : end) + 1] ==
                              ijk[3 * (int64_t)(order ? order[end - 1] : end - 1) + 1])
            ++end;
        bounds[++ns] = end;
        start = end;
    }
    return ns;
}

double trpdrv_triple_flops(int nocc, int nvir)
{
    return 16.0 * (double)nvir * (double)nvir * ((double)nvir + (double)nocc);
}

int trpdrv_tensor_a_dependent(int tensor)
{
    return tensor == TRPDRV_T_JVV || tensor == TRPDRV_T_KVV || tensor == TRPDRV_T_DINTC || tensor == TRPDRV_T_DINTX ||
           tensor == TRPDRV_T_T1V;
}

size_t trpdrv_tensor_elems(int tensor, int ncor, int nocc, int nvir)
{
    const size_t o = (size_t)(nocc > 0 ? nocc : 0), v = (size_t)(nvir > 0 ? nvir : 0);
    switch (tensor) {
    case TRPDRV_T_EORB: return (size_t)(ncor > 0 ? ncor : 0) + o + v;
    case TRPDRV_T_T2: return o * o * v * v;
    case TRPDRV_T_JVV:
    case TRPDRV_T_KVV: return o * v * v;
    case TRPDRV_T_TOV:
    case TRPDRV_T_XOV: return o * v * o;
    case TRPDRV_T_JOV:
    case TRPDRV_T_KOV: return o * o * o * v;
    case TRPDRV_T_DINTC:
    case TRPDRV_T_DINTX:
    case TRPDRV_T_T1V: return o * v;
    default: return 0;
    }
}

/* SplitMix64 finaliser (Steele, Lea & Flood, OOPSLA 2014): a counter-based stream, so element n
 * of tensor w under seed s is the same no matter how the buffer is split or threaded. */
static inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline uint64_t stream_key(uint64_t seed, int tensor)
{
    return mix64(seed ^ ((uint64_t)(tensor + 1) * 0xD1B54A32D192ED03ull));
}

static inline double unit53(uint64_t h) { return (double)(h >> 11) * 0x1.0p-53; }

static int cmp_double(const void *a, const void *b)
{
    const double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

int trpdrv_synth_fill(int tensor, int ncor, int nocc, int nvir, uint64_t seed, int dist, double *out, size_t n)
{
    if (tensor < 0 || tensor >= TRPDRV_T_COUNT || !out || ncor < 0 || nocc < 1 || nvir < 1) return TRPDRV_ERR_ARG;
    if (dist != TRPDRV_DIST_UNIFORM && dist != TRPDRV_DIST_LOGUNIFORM) return TRPDRV_ERR_ARG;
    if (n != trpdrv_tensor_elems(tensor, ncor, nocc, nvir)) return TRPDRV_ERR_ARG;
    const uint64_t key = stream_key(seed, tensor);

    if (tensor == TRPDRV_T_EORB) {
        for (size_t t = 0; t < n; ++t) {
            const double u = unit53(mix64(key + t));
            if ((int)t < ncor)
                out[t] = -20.0 + 15.0 * u;
            else if ((int)t < ncor + nocc)
                out[t] = -2.0 + 1.5 * u;
            else
                out[t] = 0.2 + 2.8 * u;
        }
        qsort(out, (size_t)ncor, sizeof(double), cmp_double);
        qsort(out + ncor, (size_t)nocc, sizeof(double), cmp_double);
        qsort(out + ncor + nocc, (size_t)nvir, sizeof(double), cmp_double);
        return TRPDRV_OK;
    }

    double half;
    int integral = 0;
    switch (tensor) {
    case TRPDRV_T_T2: half = 0.05; break;
    case TRPDRV_T_TOV:
    case TRPDRV_T_XOV:
    case TRPDRV_T_T1V: half = 0.02; break;
    default: half = 0.1; integral = 1; break;
    }
    const int logu = integral && dist == TRPDRV_DIST_LOGUNIFORM;
    const long long nn = (long long)n;
#pragma omp parallel for schedule(static)
    for (long long t = 0; t < nn; ++t) {
        const uint64_t h = mix64(key + (uint64_t)t);
        const double u = unit53(h);
        if (logu) {
            const double mag = pow(10.0, -6.0 * u); /* log-uniform magnitude in (1e-6, 1] */
            out[t] = (h & 1u) ? -mag : mag;
        } else {
            out[t] = -half + 2.0 * half * u;
        }
    }
    return TRPDRV_OK;
}
