// FP32 parity form of the triples body: the single-precision variant of the reference
// (gpu-omp/ccsd_trpdrv_omp_cbody.c:38-226, 16 cblas_sgemm calls and the float tengy loop, and
// gpu-omp/ccsd_tengy_c99.c:5-119) on the GPU, built into its own library, libtrpdrv_b200_fp32.so,
// because its entry points keep the reference's names with float arguments
// (gpu-omp/test.c:24-62).  It exists to compare with that variant's numbers, not for speed:
//
//  * sgemm_group_kernel: the eight f = A1 op(B1) - A2 B2 of one triple in IEEE FP32 (FFMA, no TF32),
//    64 x 64 output tiles, 16-index contraction chunks staged in shared memory, 4 x 4 outputs per
//    thread;
//  * tengy_f32_kernel: the (b,c) sum of the reference's float energy forms over 32 x 32 tile pairs
//    (the denominator formed as the reference forms it: -1.0 / (float sum), a double division
//    rounded to float), float partial sums per tile pair, then one block sums the pairs in a fixed
//    order.
//
// All arithmetic of the energies is float, like the reference's (its emp4i..emp5k are float).

#include <cuda_runtime.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "trpdrv_fp32.h"

namespace trpdrv {
namespace f32 {

constexpr int BT = 64;   // output tile edge
constexpr int KB = 16;   // contraction chunk
constexpr int TT = 32;   // tengy tile edge
constexpr int NT = 256;  // threads per CTA

struct GemmArgs {
    int nocc, nvir;
    const float *a1[8], *b1[8], *a2[8], *b2[8];
    int b1_t[8];  // 1: B1 enters transposed (B1'(d, c) = B1[c + d nvir])
    float *f;     // [8][nvir][nvir]
};

// f_x(b, c) = sum_d A1(b, d) B1'(d, c) - sum_m A2(b, m) B2(m, c), column-major like the reference.
__global__ void __launch_bounds__(NT) sgemm_group_kernel(const GemmArgs P)
{
    __shared__ float As[KB][BT + 4], Bs[KB][BT + 4];
    const int x = blockIdx.z, V = P.nvir, O = P.nocc;
    const int b0 = blockIdx.x * BT, c0 = blockIdx.y * BT;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4] = {};
    const float *A1 = P.a1[x], *B1 = P.b1[x], *A2 = P.a2[x], *B2 = P.b2[x];
    const int bt = P.b1_t[x];
    for (int phase = 0; phase < 2; ++phase) {
        const int K = phase ? O : V;
        for (int k0 = 0; k0 < K; k0 += KB) {
            for (int e = threadIdx.x; e < KB * BT; e += NT) {
                // A tile: rows b contiguous in memory
                const int bb = e % BT, kk = e / BT, b = b0 + bb, k = k0 + kk;
                float av = 0.0f;
                if (b < V && k < K) av = phase ? -A2[b + (size_t)k * V] : A1[b + (size_t)k * V];
                As[kk][bb] = av;
                // B tile: contiguous along c when B1 enters transposed, else along the contraction
                int cc, kb;
                if (!phase && bt) {
                    cc = e % BT;
                    kb = e / BT;
                } else {
                    kb = e % KB;
                    cc = e / KB;
                }
                const int c = c0 + cc, k2 = k0 + kb;
                float bv = 0.0f;
                if (c < V && k2 < K)
                    bv = phase ? B2[k2 + (size_t)c * O] : (bt ? B1[c + (size_t)k2 * V] : B1[k2 + (size_t)c * V]);
                Bs[kb][cc] = bv;
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < KB; ++kk) {
                float a[4], b[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    a[u] = As[kk][ty + 16 * u];
                    b[u] = Bs[kk][tx + 16 * u];
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int w = 0; w < 4; ++w) acc[u][w] = fmaf(a[u], b[w], acc[u][w]);
            }
            __syncthreads();
        }
    }
    float *F = P.f + (size_t)x * V * V;
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const int b = b0 + ty + 16 * u, c = c0 + tx + 16 * w;
            if (b < V && c < V) F[b + (size_t)c * V] = acc[u][w];
        }
}

struct TengyArgs {
    int ncor, nocc, nvir, nb;
    float eaijk;
    const float *f;  // f1n f2n f3n f4n f1t f2t f3t f4t
    const float *eorb, *dintc1, *dintx1, *t1v1, *dintc2, *dintx2, *t1v2;
    float *pair;     // [npairs][4]
};

// the reference's float forms at one (b, c): gpu-omp/ccsd_trpdrv_omp_cbody.c:176-217
__device__ __forceinline__ void term(const TengyArgs &P, int b, int c, float (&s)[4])
{
    const int V = P.nvir;
    const size_t vv = (size_t)V * V, bc = b + (size_t)c * V, cb = c + (size_t)b * V;
    const float *f = P.f;
    const float e_b = P.eorb[P.ncor + P.nocc + b], e_c = P.eorb[P.ncor + P.nocc + c];
    const float denom = (float)(-1.0 / (double)(e_b + e_c + P.eaijk));
    const float n1bc = f[bc], n2bc = f[vv + bc], n3bc = f[2 * vv + bc], n4bc = f[3 * vv + bc];
    const float t1bc = f[4 * vv + bc], t2bc = f[5 * vv + bc], t3bc = f[6 * vv + bc], t4bc = f[7 * vv + bc];
    const float n1cb = f[cb], n2cb = f[vv + cb], n3cb = f[2 * vv + cb], n4cb = f[3 * vv + cb];
    const float t1cb = f[4 * vv + cb], t2cb = f[5 * vv + cb], t3cb = f[6 * vv + cb], t4cb = f[7 * vv + cb];
    s[0] += denom * (t1bc + n1cb + t2cb + n3bc + n4cb) * (t1bc - t2bc * 2 - t3bc * 2 + t4bc)
          - denom * (n1bc + t1cb + n2cb + n3cb) * (t1bc * 2 - t2bc - t3bc + t4bc * 2)
          + denom * 3 * (n1bc * (n1bc + n3cb + t4cb * 2) + n2bc * t2cb + n3bc * t4bc);
    s[2] += denom * (n1bc + t1cb + n2cb + t3bc + t4cb) * (n1bc - n2bc * 2 - n3bc * 2 + n4bc)
          - denom * (t1bc + n1cb + t2cb + t3cb) * (n1bc * 2 - n2bc - n3bc + n4bc * 2)
          + denom * 3 * (t1bc * (t1bc + t3cb + n4cb * 2) + t2bc * n2cb + t3bc * n4bc);
    const float t1v1b = P.t1v1[b], t1v2b = P.t1v2[b];
    const float dx1c = P.dintx1[c], dx2c = P.dintx2[c], dc1c = P.dintc1[c], dc2c = P.dintc2[c];
    s[1] += denom * t1v1b * dx1c * (t1bc + n2bc + n4cb - (t3bc + n4bc + n2cb + n1bc + t2bc + n3cb) * 2
                                    + (n3bc + t4bc + n1cb) * 4)
          + denom * t1v1b * dc1c * (n1bc + n4bc + t1cb - (n2bc + n3bc + t2cb) * 2);
    s[3] += denom * t1v2b * dx2c * (n1bc + t2bc + t4cb - (n3bc + t4bc + t2cb + t1bc + n2bc + t3cb) * 2
                                    + (t3bc + n4bc + t1cb) * 4)
          + denom * t1v2b * dc2c * (t1bc + t4bc + n1cb - (t2bc + t3bc + n2cb) * 2);
}

// one CTA per 32 x 32 tile pair (B <= C); the pair's sums over (b, c) in B x C and, for B < C, C x B
__global__ void __launch_bounds__(NT) tengy_f32_kernel(const TengyArgs P)
{
    __shared__ float red[4][NT / 32];
    int B = 0, rem = blockIdx.x;
    while (rem >= P.nb - B) {
        rem -= P.nb - B;
        ++B;
    }
    const int C = B + rem, V = P.nvir;
    float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int e = threadIdx.x; e < TT * TT; e += NT) {
        const int b = B * TT + (e & 31), c = C * TT + (e >> 5);
        if (b < V && c < V) {
            term(P, b, c, s);
            if (B != C) term(P, c, b, s);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float v = s[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        float v = 0.0f;
        for (int w = 0; w < NT / 32; ++w) v += red[threadIdx.x][w];
        P.pair[4 * blockIdx.x + threadIdx.x] = v;
    }
}

// the tile pairs' sums in a fixed order: out[0..3] = emp4i, emp5i, emp4k, emp5k
__global__ void pair_sum_kernel(const float *pair, int npairs, float *out)
{
    if (threadIdx.x < 4) {
        float v = 0.0f;
        for (int p = 0; p < npairs; ++p) v += pair[4 * p + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

// ------------------------------------------------------------------------------------------------
// host state: one device, one stream, buffers grown to the largest shape seen
// ------------------------------------------------------------------------------------------------
enum { S_TIJ, S_TKJ, S_JIA, S_JKA, S_KIA, S_KKA, S_NVV };
enum { O_TIA, O_TKA, O_XIA, O_XKA, O_JIJ, O_JKJ, O_KIJ, O_KKJ, O_NOV };

struct State {
    int ready;
    cudaStream_t st;
    size_t cap_vv, cap_ov, cap_v, cap_bf, cap_pairs;
    float *vv[S_NVV], *ov[O_NOV], *vec[6], *eorb, *f, *pair, *out;
    float *h_out;  // pinned, 4 floats
};
State g;
pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;
thread_local char t_msg[256];
thread_local int t_status;

int fail(int status, const char *msg)
{
    snprintf(t_msg, sizeof t_msg, "%s", msg);
    t_status = status;
    return status;
}

#define F32_TRY(call)                                                                   \
    do {                                                                                \
        const cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) {                                                        \
            char m_[200];                                                               \
            snprintf(m_, sizeof m_, "%s: %s", #call, cudaGetErrorString(e_));          \
            return fail(e_ == cudaErrorMemoryAllocation ? 3 : 2, m_);                   \
        }                                                                               \
    } while (0)

int grow(float **p, size_t *cap, size_t want)
{
    if (want <= *cap) return 0;
    if (*p) cudaFree(*p);
    *p = nullptr;
    F32_TRY(cudaMalloc((void **)p, sizeof(float) * want));
    *cap = want;
    return 0;
}

int reserve(int nocc, int nvir, int nbf)
{
    if (!g.ready) {
        int dev = 0, major = 0;
        F32_TRY(cudaGetDevice(&dev));
        F32_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
        if (major != 10) return fail(4, "the current device is not sm_100");
        F32_TRY(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
        F32_TRY(cudaMalloc((void **)&g.out, sizeof(float) * 4));
        F32_TRY(cudaMallocHost((void **)&g.h_out, sizeof(float) * 4));
        g.ready = 1;
    }
    const size_t vv = (size_t)nvir * nvir, ov = (size_t)nocc * nvir, v = (size_t)nvir;
    const int nb = (nvir + TT - 1) / TT;
    const size_t pairs = (size_t)nb * (nb + 1) / 2;
    if (vv > g.cap_vv) {
        size_t c = 0;
        for (int q = 0; q < S_NVV; ++q) {
            c = 0;
            if (g.vv[q]) cudaFree(g.vv[q]);
            g.vv[q] = nullptr;
            if (grow(&g.vv[q], &c, vv)) return t_status;
        }
        c = 0;
        if (g.f) cudaFree(g.f);
        g.f = nullptr;
        if (grow(&g.f, &c, 8 * vv)) return t_status;
        g.cap_vv = vv;
    }
    if (ov > g.cap_ov) {
        for (int q = 0; q < O_NOV; ++q) {
            size_t c = 0;
            if (g.ov[q]) cudaFree(g.ov[q]);
            g.ov[q] = nullptr;
            if (grow(&g.ov[q], &c, ov)) return t_status;
        }
        g.cap_ov = ov;
    }
    if (v > g.cap_v) {
        for (int q = 0; q < 6; ++q) {
            size_t c = 0;
            if (g.vec[q]) cudaFree(g.vec[q]);
            g.vec[q] = nullptr;
            if (grow(&g.vec[q], &c, v)) return t_status;
        }
        g.cap_v = v;
    }
    if (grow(&g.eorb, &g.cap_bf, (size_t)nbf)) return t_status;
    if (grow(&g.pair, &g.cap_pairs, 4 * pairs)) return t_status;
    return 0;
}

int h2d(float *dst, const float *src, size_t n)
{
    F32_TRY(cudaMemcpyAsync(dst, src, sizeof(float) * n, cudaMemcpyHostToDevice, g.st));
    return 0;
}

int launch_tengy(int ncor, int nocc, int nvir, float eaijk, const float *f, const float *const *vec,
                 const float *eorb, float *out4)
{
    TengyArgs T;
    T.ncor = ncor;
    T.nocc = nocc;
    T.nvir = nvir;
    T.nb = (nvir + TT - 1) / TT;
    T.eaijk = eaijk;
    T.f = f;
    T.eorb = eorb;
    T.dintc1 = vec[0];
    T.dintx1 = vec[1];
    T.t1v1 = vec[2];
    T.dintc2 = vec[3];
    T.dintx2 = vec[4];
    T.t1v2 = vec[5];
    T.pair = g.pair;
    const int npairs = T.nb * (T.nb + 1) / 2;
    tengy_f32_kernel<<<npairs, NT, 0, g.st>>>(T);
    pair_sum_kernel<<<1, 32, 0, g.st>>>(g.pair, npairs, g.out);
    F32_TRY(cudaGetLastError());
    F32_TRY(cudaMemcpyAsync(g.h_out, g.out, sizeof(float) * 4, cudaMemcpyDeviceToHost, g.st));
    F32_TRY(cudaStreamSynchronize(g.st));
    for (int q = 0; q < 4; ++q) out4[q] = g.h_out[q];
    return 0;
}

int body(float *f1n, float *f1t, float *f2n, float *f2t, float *f3n, float *f3t, float *f4n, float *f4t,
         const float *eorb, const int *ncor_, const int *nocc_, const int *nvir_, float *emp4_, float *emp5_,
         const int *a_, const int *i_, const int *j_, const int *k_, const int *klo_, const float *tij,
         const float *tkj, const float *tia, const float *tka, const float *xia, const float *xka, const float *jia,
         const float *jka, const float *kia, const float *kka, const float *jij, const float *jkj, const float *kij,
         const float *kkj, const float *dintc1, const float *dintx1, const float *t1v1, const float *dintc2,
         const float *dintx2, const float *t1v2)
{
    if (!ncor_ || !nocc_ || !nvir_ || !a_ || !i_ || !j_ || !k_ || !klo_ || !emp4_ || !emp5_ || !eorb)
        return fail(1, "NULL argument");
    const int ncor = *ncor_, nocc = *nocc_, nvir = *nvir_, a = *a_, i = *i_, j = *j_, k = *k_, klo = *klo_;
    const float *arr[] = {tij, tkj, tia, tka, xia, xka, jia, jka, kia, kka, jij, jkj, kij, kkj,
                          dintc1, dintx1, t1v1, dintc2, dintx2, t1v2};
    for (const float *p : arr)
        if (!p) return fail(1, "NULL array argument");
    if (nocc < 1 || nvir < 1 || ncor < 0 || nocc > 1023 || nvir > 16384) return fail(1, "ncor/nocc/nvir out of range");
    const int nbf = ncor + nocc + nvir;
    if (a < 1 || a > nbf || i < 1 || i > nocc || j < 1 || j > nocc || k < 1 || k > nocc || klo < 1 || klo > k)
        return fail(1, "orbital index out of range");
    const char *wf = getenv("TRPDRV_WRITE_F");
    const int write_f = wf && strcmp(wf, "1") == 0;
    if (write_f && (!f1n || !f1t || !f2n || !f2t || !f3n || !f3t || !f4n || !f4t))
        return fail(1, "TRPDRV_WRITE_F=1 with a NULL f array");
    if (int rc = reserve(nocc, nvir, nbf)) return rc;
    const size_t vv = (size_t)nvir * nvir, ov = (size_t)nocc * nvir;
    const size_t kv = (size_t)(k - klo) * vv, ko = (size_t)(k - klo) * ov;
    // the reference's offsets of the k-chunk slices (gpu-omp/ccsd_trpdrv_omp_cbody.c:64-70)
    const float *svv[S_NVV] = {tij, tkj + kv, jia, jka + kv, kia, kka + kv};
    const float *sov[O_NOV] = {tia, tka + ko, xia, xka + ko, jij, jkj + ko, kij, kkj + ko};
    const float *svec[6] = {dintc1, dintx1, t1v1, dintc2, dintx2, t1v2};
    for (int q = 0; q < S_NVV; ++q)
        if (int rc = h2d(g.vv[q], svv[q], vv)) return rc;
    for (int q = 0; q < O_NOV; ++q)
        if (int rc = h2d(g.ov[q], sov[q], ov)) return rc;
    for (int q = 0; q < 6; ++q)
        if (int rc = h2d(g.vec[q], svec[q], (size_t)nvir)) return rc;
    if (int rc = h2d(g.eorb, eorb, (size_t)nbf)) return rc;

    // f1n f2n f3n f4n f1t f2t f3t f4t: gpu-omp/ccsd_trpdrv_omp_cbody.c:72-167
    GemmArgs G;
    G.nocc = nocc;
    G.nvir = nvir;
    G.f = g.f;
    float *const *V = g.vv, *const *Ob = g.ov;
    const float *a1[8] = {V[S_JIA], V[S_KIA], V[S_JIA], V[S_KIA], V[S_JKA], V[S_KKA], V[S_JKA], V[S_KKA]};
    const float *b1[8] = {V[S_TKJ], V[S_TKJ], V[S_TKJ], V[S_TKJ], V[S_TIJ], V[S_TIJ], V[S_TIJ], V[S_TIJ]};
    const int bt[8] = {1, 1, 0, 0, 1, 1, 0, 0};
    const float *a2[8] = {Ob[O_TIA], Ob[O_XIA], Ob[O_TIA], Ob[O_XIA], Ob[O_TKA], Ob[O_XKA], Ob[O_TKA], Ob[O_XKA]};
    const float *b2[8] = {Ob[O_KKJ], Ob[O_KKJ], Ob[O_JKJ], Ob[O_JKJ], Ob[O_KIJ], Ob[O_KIJ], Ob[O_JIJ], Ob[O_JIJ]};
    for (int x = 0; x < 8; ++x) {
        G.a1[x] = a1[x];
        G.b1[x] = b1[x];
        G.b1_t[x] = bt[x];
        G.a2[x] = a2[x];
        G.b2[x] = b2[x];
    }
    const dim3 grid((nvir + BT - 1) / BT, (nvir + BT - 1) / BT, 8);
    sgemm_group_kernel<<<grid, NT, 0, g.st>>>(G);
    F32_TRY(cudaGetLastError());

    // gpu-omp/ccsd_trpdrv_omp_cbody.c:62
    const float eaijk = eorb[a - 1] - (eorb[ncor + i - 1] + eorb[ncor + j - 1] + eorb[ncor + k - 1]);
    const float *dvec[6] = {g.vec[0], g.vec[1], g.vec[2], g.vec[3], g.vec[4], g.vec[5]};
    float r[4];
    if (int rc = launch_tengy(ncor, nocc, nvir, eaijk, g.f, dvec, g.eorb, r)) return rc;
    if (write_f) {
        float *outs[8] = {f1n, f2n, f3n, f4n, f1t, f2t, f3t, f4t};
        for (int x = 0; x < 8; ++x)
            F32_TRY(cudaMemcpy(outs[x], g.f + (size_t)x * vv, sizeof(float) * vv, cudaMemcpyDeviceToHost));
    }
    // gpu-omp/ccsd_trpdrv_omp_cbody.c:220-228
    float emp4 = *emp4_, emp5 = *emp5_;
    emp4 += r[0];
    emp5 += r[1];
    if (*i_ != *k_) {
        emp4 += r[2];
        emp5 += r[3];
    }
    *emp4_ = emp4;
    *emp5_ = emp5;
    return 0;
}

int tengy(const float *const *f8, const float *const *vec, const float *eorb, float eaijk, float *out4, int ncor,
          int nocc, int nvir)
{
    for (int q = 0; q < 8; ++q)
        if (!f8[q]) return fail(1, "NULL f array");
    for (int q = 0; q < 6; ++q)
        if (!vec[q]) return fail(1, "NULL vector");
    if (!eorb || nocc < 1 || nvir < 1 || ncor < 0 || nvir > 16384) return fail(1, "bad tengy arguments");
    const int nbf = ncor + nocc + nvir;
    if (int rc = reserve(nocc, nvir, nbf)) return rc;
    const size_t vv = (size_t)nvir * nvir;
    // device order f1n f2n f3n f4n f1t f2t f3t f4t from the argument order f1n f1t f2n f2t ...
    for (int x = 0; x < 4; ++x) {
        if (int rc = h2d(g.f + (size_t)x * vv, f8[2 * x], vv)) return rc;
        if (int rc = h2d(g.f + (size_t)(4 + x) * vv, f8[2 * x + 1], vv)) return rc;
    }
    for (int q = 0; q < 6; ++q)
        if (int rc = h2d(g.vec[q], vec[q], (size_t)nvir)) return rc;
    if (int rc = h2d(g.eorb, eorb, (size_t)nbf)) return rc;
    const float *dvec[6] = {g.vec[0], g.vec[1], g.vec[2], g.vec[3], g.vec[4], g.vec[5]};
    return launch_tengy(ncor, nocc, nvir, eaijk, g.f, dvec, g.eorb, out4);
}

void report(int rc, const char *who)
{
    if (!rc) return;
    const char *v = getenv("TRPDRV_ON_ERROR");
    if (v && strcmp(v, "return") == 0) return;
    fprintf(stderr, "%s: %s\n", who, t_msg);
    abort();
}

}  // namespace f32
}  // namespace trpdrv

using namespace trpdrv::f32;

#define F32_BODY_ARGS                                                                                       \
    float *f1n, float *f1t, float *f2n, float *f2t, float *f3n, float *f3t, float *f4n, float *f4t,        \
        float *eorb, int *ncor, int *nocc, int *nvir, float *emp4, float *emp5, int *a, int *i, int *j,    \
        int *k, int *klo, float *tij, float *tkj, float *tia, float *tka, float *xia, float *xka,           \
        float *jia, float *jka, float *kia, float *kka, float *jij, float *jkj, float *kij, float *kkj,     \
        float *dintc1, float *dintx1, float *t1v1, float *dintc2, float *dintx2, float *t1v2
#define F32_BODY_PASS                                                                                       \
    f1n, f1t, f2n, f2t, f3n, f3t, f4n, f4t, eorb, ncor, nocc, nvir, emp4, emp5, a, i, j, k, klo, tij, tkj,  \
        tia, tka, xia, xka, jia, jka, kia, kka, jij, jkj, kij, kkj, dintc1, dintx1, t1v1, dintc2, dintx2, t1v2

static void body_entry(const char *who, F32_BODY_ARGS)
{
    pthread_mutex_lock(&g_mu);
    t_status = 0;
    const int rc = body(F32_BODY_PASS);
    pthread_mutex_unlock(&g_mu);
    report(rc, who);
}

extern "C" void ccsd_trpdrv_omp_cbody_(F32_BODY_ARGS) { body_entry("ccsd_trpdrv_omp_cbody_", F32_BODY_PASS); }
extern "C" void ccsd_trpdrv_omp_fbody_(F32_BODY_ARGS) { body_entry("ccsd_trpdrv_omp_fbody_", F32_BODY_PASS); }

extern "C" void ccsd_tengy_omp(const float *f1n, const float *f1t, const float *f2n, const float *f2t,
                               const float *f3n, const float *f3t, const float *f4n, const float *f4t,
                               const float *dintc1, const float *dintx1, const float *t1v1, const float *dintc2,
                               const float *dintx2, const float *t1v2, const float *eorb, const float eaijk,
                               float *emp4i, float *emp5i, float *emp4k, float *emp5k, const int ncor,
                               const int nocc, const int nvir)
{
    pthread_mutex_lock(&g_mu);
    t_status = 0;
    int rc = (emp4i && emp5i && emp4k && emp5k) ? 0 : fail(1, "NULL output");
    const float *f8[8] = {f1n, f1t, f2n, f2t, f3n, f3t, f4n, f4t};
    const float *vec[6] = {dintc1, dintx1, t1v1, dintc2, dintx2, t1v2};
    float r[4];
    if (!rc) rc = tengy(f8, vec, eorb, eaijk, r, ncor, nocc, nvir);
    pthread_mutex_unlock(&g_mu);
    if (!rc) {  // outputs overwritten, gpu-omp/ccsd_tengy_c99.c:115-118
        *emp4i = r[0];
        *emp5i = r[1];
        *emp4k = r[2];
        *emp5k = r[3];
    }
    report(rc, "ccsd_tengy_omp");
}

extern "C" int trpdrv_fp32_last_error(void) { return t_status; }
extern "C" const char *trpdrv_fp32_last_error_message(void) { return t_msg; }
