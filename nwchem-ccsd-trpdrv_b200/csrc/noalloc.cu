// The triples body on caller-owned device buffers without any device allocation.
//
// Some callers cannot call cudaMalloc when they need this work: a host application (a quantum-
// chemistry code, for one) that reserves the device memory up front in its own pool and hands
// libraries a fixed budget, so an allocation behind its back could fail or break that budget; a
// plug-in running inside a framework that owns every device buffer; or a loop that cannot pay for
// cudaMalloc/cudaFree, which may synchronise the device, on every call.  For them,
// trpdrv_body_device_noalloc runs the plain per-triple path (the grouped FP64 GEMM that forms the
// eight f and the tengy reduction, the same kernels as the plain plans) with all of its scratch in
// one statically sized device array that the CUDA module reserves when it loads:
//
//   * at most TRPDRV_NOALLOC_MAX_NVIR virtual and TRPDRV_NOALLOC_MAX_NOCC occupied orbitals;
//   * every GPU that loads the library keeps the array (about 4.7 MB) until the process exits;
//   * all calls on a device share it, so calls that overlap on the GPU (different streams, or
//     different host threads) race on it and produce garbage: serialise them;
//   * the first call on each device looks up the array's device address (cudaGetSymbolAddress)
//     and sets the kernels' shared-memory limits; make that first call before any stream capture.
//
// The caller passes device pointers for the inputs (already sliced for the triple) and for the
// four outputs; this function enqueues on the caller's stream and returns without waiting.  It
// refuses to start while an earlier CUDA error is pending on the thread (it would otherwise read
// and clear that error as its own), and reports it without clearing it.

#include <cuda_runtime.h>
#include <pthread.h>
#include <stdio.h>

#include "launch.h"
#include "trpdrv.h"

extern "C" int trpdrv_plain_init(void);

namespace {

constexpr int MAXV = TRPDRV_NOALLOC_MAX_NVIR;
constexpr int MAXO = TRPDRV_NOALLOC_MAX_NOCC;
constexpr int MAXNB = (MAXV + TRPDRV_TILE - 1) / TRPDRV_TILE;
constexpr int MAXPAIRS = MAXNB * (MAXNB + 1) / 2;

// scratch layout (doubles): [counter block][tengy partials][4 negated occupied operands][8 f tiles]
constexpr size_t OFF_COUNTER = 0;                                  // one unsigned int, 256-byte block
constexpr size_t OFF_PARTIAL = 32;                                 // 4 * MAXPAIRS doubles
constexpr size_t OFF_NEG = OFF_PARTIAL + ((4 * MAXPAIRS + 31) / 32) * 32;
constexpr size_t OFF_F = OFF_NEG + 4 * (size_t)MAXV * MAXO;
constexpr size_t SCRATCH_DOUBLES = OFF_F + 8 * (size_t)MAXV * MAXV;

static __device__ __align__(256) double g_noalloc_scratch[SCRATCH_DOUBLES];

constexpr int MAX_DEVICES = 64;
pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;
double *g_scratch_addr[MAX_DEVICES];  // device address of g_noalloc_scratch, per device

int fail(int status, const char *msg) { return trpdrv_record_error(status, msg); }

// Once per device, with that device current: the array's device address and the kernel attributes.
int setup_device(int dev, double **out)
{
    pthread_mutex_lock(&g_mu);
    int rc = TRPDRV_OK;
    if (!g_scratch_addr[dev]) {
        double *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            char msg[256];
            snprintf(msg, sizeof msg, "trpdrv_body_device_noalloc: cudaGetSymbolAddress failed: %s",
                     cudaGetErrorString(e));
            rc = fail(TRPDRV_ERR_CUDA, msg);
        } else if (trpdrv_plain_init() != 0) {
            rc = fail(TRPDRV_ERR_CUDA, "trpdrv_body_device_noalloc: kernel attribute setup failed");
        } else {
            g_scratch_addr[dev] = p;
        }
    }
    *out = g_scratch_addr[dev];
    pthread_mutex_unlock(&g_mu);
    return rc;
}

}  // namespace

extern "C" int trpdrv_body_device_noalloc(const trpdrv_body_device_args *a, void *stream)
{
    if (!a) return fail(TRPDRV_ERR_ARG, "trpdrv_body_device_noalloc: NULL arguments");
    const int O = a->nocc, V = a->nvir;
    if (V < 1 || O < 1 || a->ncor < 0)
        return fail(TRPDRV_ERR_ARG, "trpdrv_body_device_noalloc: ncor/nocc/nvir out of range");
    if (V > MAXV || O > MAXO) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "trpdrv_body_device_noalloc: nvir=%d nocc=%d exceed the static scratch limits nvir<=%d nocc<=%d", V,
                 O, MAXV, MAXO);
        return fail(TRPDRV_ERR_ARG, msg);
    }
    const int nbf = a->ncor + O + V;
    if (a->a < 1 || a->a > nbf || a->i < 1 || a->i > O || a->j < 1 || a->j > O || a->k < 1 || a->k > O)
        return fail(TRPDRV_ERR_ARG, "trpdrv_body_device_noalloc: orbital index out of range");
    const double *in[] = {a->eorb, a->tij, a->tkj, a->tia, a->tka, a->xia, a->xka, a->jia, a->jka, a->kia, a->kka,
                          a->jij, a->jkj, a->kij, a->kkj, a->dintc1, a->dintx1, a->t1v1, a->dintc2, a->dintx2, a->t1v2};
    for (const double *p : in)
        if (!p) return fail(TRPDRV_ERR_ARG, "trpdrv_body_device_noalloc: NULL input pointer");
    if (!a->out4) return fail(TRPDRV_ERR_ARG, "trpdrv_body_device_noalloc: NULL output pointer");

    // an error left by the caller's earlier work stays the caller's: report it, do not clear it
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof msg, "trpdrv_body_device_noalloc: an earlier CUDA error is pending (%s); nothing enqueued",
                 cudaGetErrorString(pending));
        return fail(TRPDRV_ERR_STATE, msg);
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return fail(TRPDRV_ERR_NODEV, "trpdrv_body_device_noalloc: no current CUDA device");
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (major != 10 || minor != 0)
        return fail(TRPDRV_ERR_NODEV, "trpdrv_body_device_noalloc: the current device is not sm_100");
    double *scratch = nullptr;
    const int rc = setup_device(dev, &scratch);
    if (rc != TRPDRV_OK) return rc;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + OFF_COUNTER);
    double *partial = scratch + OFF_PARTIAL;
    double *neg = scratch + OFF_NEG;
    double *f = scratch + OFF_F;
    const size_t lnov = (size_t)O * V;

    // the last CTA of the reduction must see a zero counter, whatever a previous call left behind
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return fail(TRPDRV_ERR_CUDA, "trpdrv_body_device_noalloc: clearing the counter failed");
    // -tia, -xia, -tka, -xka (the reference's alpha = -1 GEMMs, omp/ccsd_trpdrv_omp_cbody.c:73-116)
    const double *occ[4] = {a->tia, a->xia, a->tka, a->xka};
    for (int q = 0; q < 4; ++q)
        if (trpdrv_launch_negate(occ[q], neg + q * lnov, lnov, st) != 0)
            return fail(TRPDRV_ERR_CUDA, "trpdrv_body_device_noalloc: launch failed");

    trpdrv_plain_args ga = {};
    ga.nocc = O;
    ga.nvir = V;
    ga.f = f;
    const double *nt_i = neg, *nx_i = neg + lnov, *nt_k = neg + 2 * lnov, *nx_k = neg + 3 * lnov;
    // f1n f2n f3n f4n f1t f2t f3t f4t: omp/ccsd_trpdrv_omp_cbody.c:70-117
    const double *a1[8] = {a->jia, a->kia, a->jia, a->kia, a->jka, a->kka, a->jka, a->kka};
    const double *b1[8] = {a->tkj, a->tkj, a->tkj, a->tkj, a->tij, a->tij, a->tij, a->tij};
    const int nt[8] = {1, 1, 0, 0, 1, 1, 0, 0};
    const double *a2[8] = {nt_i, nx_i, nt_i, nx_i, nt_k, nx_k, nt_k, nx_k};
    const double *b2[8] = {a->kkj, a->kkj, a->jkj, a->jkj, a->kij, a->kij, a->jij, a->jij};
    int vec2 = !(V & 1) && !(O & 1);
    for (int x = 0; x < 8; ++x) {
        ga.a1[x] = a1[x];
        ga.b1[x] = b1[x];
        ga.b1_nt[x] = nt[x];
        ga.a2[x] = a2[x];
        ga.b2[x] = b2[x];
        const double *ops[4] = {a1[x], b1[x], a2[x], b2[x]};
        for (const double *p : ops)
            if (reinterpret_cast<uintptr_t>(p) & 15u) vec2 = 0;  // 16-byte copies need 16-byte alignment
    }
    if (trpdrv_launch_plain_gemm(&ga, vec2, st) != 0)
        return fail(TRPDRV_ERR_CUDA, "trpdrv_body_device_noalloc: launch failed");

    trpdrv_tengy_args ta = {};
    ta.ncor = a->ncor;
    ta.nocc = O;
    ta.nvir = V;
    ta.use_eaijk = 0;  // eaijk from eorb and a, i, j, k on the device (omp/ccsd_trpdrv_omp_cbody.c:126)
    ta.a = a->a;
    ta.i = a->i;
    ta.j = a->j;
    ta.k = a->k;
    ta.f = f;
    ta.eorb = a->eorb;
    ta.dintc1 = a->dintc1;
    ta.dintx1 = a->dintx1;
    ta.t1v1 = a->t1v1;
    ta.dintc2 = a->dintc2;
    ta.dintx2 = a->dintx2;
    ta.t1v2 = a->t1v2;
    ta.block_partial = partial;
    ta.counter = counter;
    ta.out4 = a->out4;
    if (trpdrv_launch_tengy(&ta, st) != 0) return fail(TRPDRV_ERR_CUDA, "trpdrv_body_device_noalloc: launch failed");
    return TRPDRV_OK;
}
