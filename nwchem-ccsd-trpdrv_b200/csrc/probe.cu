// Issue-rate probes: the roofline denominators for the FP64 contraction kernels and the int8 form.
//
// A measurement tool, not part of the product: it is built into its own library,
// lib/libtrpdrv_probe.so, which only the benchmark loads.
//
// FP64: every warp keeps NACC independent accumulator chains in registers and issues NACC MMAs (or
// DFMAs) per iteration with register operands only, so the measured rate is the FP64 tensor (or FMA)
// pipe throughput of the device, not a memory rate.  The accumulators are written out at the end so
// the work cannot be eliminated.
//
// int8: one thread per SM issues tcgen05.mma.kind::i8 (M = 128, K = 32, N = 64 / 128 / 256) from
// digit-like operands in shared memory in the emulated form's order: 7 A slices x 7 B slices with
// p + q < 7, A slice p shared by its 7 - p products through the A collector, level p + q accumulating
// in tensor memory.  Nothing is loaded from HBM, so the rate is the tensor pipe's for that
// instruction shape.

#include "device_common.cuh"
#include <cuda_runtime.h>

namespace trpdrv {
namespace probe {

constexpr int NACC = 8;
constexpr int NTHREAD = 256;

template <int KIND>
__global__ void __launch_bounds__(NTHREAD)
probe_kernel(int iters, double *sink)
{
    // every operand register distinct: repeated registers inside one MMA understate the rate
    double a[8], b[4];
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = 1.0 + 1e-9 * (threadIdx.x + q);
#pragma unroll
    for (int q = 0; q < 4; ++q) b[q] = 0.5 + 1e-9 * (threadIdx.x + 3 * q);
    double acc[NACC][4];
#pragma unroll
    for (int q = 0; q < NACC; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[q][e] = 0.0;
    const double (&a4)[4] = *reinterpret_cast<const double(*)[4]>(a);
    const double (&b2)[2] = *reinterpret_cast<const double(*)[2]>(b);

    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < NACC; ++q) {
            if (KIND == 0) {
                double d[2] = {acc[q][0], acc[q][1]};
                dmma_8x8x4(d, a[0], b[0]);
                acc[q][0] = d[0];
                acc[q][1] = d[1];
            } else if (KIND == 1) {
                dmma_16x8x4(acc[q], a[0], a[1], b[0]);
            } else if (KIND == 2) {
                dmma_16x8x8(acc[q], a4, b2);
            } else if (KIND == 3) {
                dmma_16x8x16(acc[q], a, b);
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) asm volatile("fma.rn.f64 %0, %1, %2, %0;" : "+d"(acc[q][e]) : "d"(a[e]), "d"(b[e]));
            }
        }
    }
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < NACC; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e) s += acc[q][e];
    sink[blockIdx.x * NTHREAD + threadIdx.x] = s;
}

// ---- int8 tcgen05 issue rate --------------------------------------------------------------------
constexpr int I8_S = 7;              // digit slices: 28 products per k-step
constexpr int I8_KC = 64;            // bytes of K per operand row (two 32-wide k-steps)
constexpr int I8_SMEM = 200 * 1024;  // dynamic shared memory: one CTA per SM
constexpr unsigned long long I8_WAIT_NS = 4000000000ull;

__device__ __forceinline__ unsigned i8_saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long i8_timer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// K-major operand rows of 64 bytes with the 64-byte swizzle: 8-row atoms of 512 bytes, version 1
__device__ __forceinline__ unsigned long long i8_desc(const void *p)
{
    return (unsigned long long)((i8_saddr(p) >> 4) & 0x3FFFu) | (1ull << 16) | ((unsigned long long)(512 >> 4) << 32) |
           (1ull << 46) | (4ull << 61);
}

// kind::i8 instruction descriptor: D s32, A and B signed, both K-major, N >> 3, M >> 4
template <int M, int N>
__host__ __device__ constexpr unsigned i8_idesc()
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(M >> 4) << 24);
}

template <int N, bool PAIR, int COL>
__device__ __forceinline__ void i8_mma(unsigned d, unsigned long long a, unsigned long long b)
{
#define PROBE_I8_MMA1(Q)                                                                                           \
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::i8" Q              \
                 " [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(d),                                         \
                 "l"(a), "l"(b), "r"(i8_idesc<128, N>()), "r"(1), "r"(0)                                          \
                 : "memory")
#define PROBE_I8_MMA2(Q)                                                                                           \
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::2.kind::i8" Q              \
                 " [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n}\n" ::"r"(d),                         \
                 "l"(a), "l"(b), "r"(i8_idesc<256, N>()), "r"(1), "r"(0)                                          \
                 : "memory")
    if constexpr (!PAIR) {
        if (COL == 1)
            PROBE_I8_MMA1(".collector::a::fill");
        else if (COL == 2)
            PROBE_I8_MMA1(".collector::a::use");
        else if (COL == 3)
            PROBE_I8_MMA1(".collector::a::lastuse");
        else
            PROBE_I8_MMA1("");
    } else {
        if (COL == 1)
            PROBE_I8_MMA2(".collector::a::fill");
        else if (COL == 2)
            PROBE_I8_MMA2(".collector::a::use");
        else if (COL == 3)
            PROBE_I8_MMA2(".collector::a::lastuse");
        else
            PROBE_I8_MMA2("");
    }
#undef PROBE_I8_MMA1
#undef PROBE_I8_MMA2
}

// the products of one k-step, A slice P with B slices Q.. (p-major, collector over each A slice)
template <int N, bool PAIR, int P, int Q>
__device__ __forceinline__ void i8_kstep(unsigned tmem, unsigned long long dA, unsigned long long dB, int ks)
{
    if constexpr (P < I8_S) {
        if constexpr (Q < I8_S - P) {
            constexpr int n = I8_S - P, NLEV = 512 / N < I8_S ? 512 / N : I8_S;
            constexpr int col = n == 1 ? 0 : Q == 0 ? 1 : Q == n - 1 ? 3 : 2;
            // A slice P at P x 8 KB, B slice Q at Q x (N x 64) bytes; descriptors count 16-byte units
            i8_mma<N, PAIR, col>(tmem + (unsigned)(((P + Q) % NLEV) * N), dA + (unsigned long long)(P * 512 + ks * 2),
                                 dB + (unsigned long long)(Q * (N * I8_KC / 16) + ks * 2));
            i8_kstep<N, PAIR, P, Q + 1>(tmem, dA, dB, ks);
        } else {
            i8_kstep<N, PAIR, P + 1, 0>(tmem, dA, dB, ks);
        }
    }
}

__device__ __forceinline__ bool i8_try_wait(unsigned long long *b, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(i8_saddr(b)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// bounded wait (I8_WAIT_NS); false when it ran out
__device__ __forceinline__ bool i8_wait(unsigned long long *b, unsigned parity)
{
    const unsigned long long t0 = i8_timer();
    while (!i8_try_wait(b, parity))
        if (i8_timer() - t0 > I8_WAIT_NS) return false;
    return true;
}

__device__ __forceinline__ void i8_cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// PAIR: a cluster of two CTAs on two SMs; the even CTA issues cta_group::2 MMAs with M = 256 (each
// CTA holding 128 rows of A and its TMEM levels) and the completion is multicast to both CTAs.
// HS: the issuer works in chunks of two k-steps behind a two-stage ring (wait full, 56 MMAs, commit
// empty) that a second thread re-arms, as the contraction kernel's MMA warp and producer do, minus the
// copies.
template <int N, bool PAIR, bool HS>
__global__ void __launch_bounds__(128, 1) int8_probe_kernel(int iters, int *status)
{
    static_assert(!(PAIR && HS), "the handshake form commits per CTA: single-SM only");
    extern __shared__ __align__(1024) unsigned char i8_raw[];
    constexpr int A_BYTES = I8_S * 128 * I8_KC, B_BYTES = I8_S * N * I8_KC;
    static_assert(A_BYTES + B_BYTES + 1024 + 64 <= I8_SMEM, "operands exceed the probe's shared memory");
    unsigned char *sm = i8_raw + ((1024u - (i8_saddr(i8_raw) & 1023u)) & 1023u);
    // after the operands: done, the TMEM slot (4 bytes in the second word), full[2], empty[2]
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(sm + A_BYTES + B_BYTES);
    unsigned *tslot = reinterpret_cast<unsigned *>(bar + 1);
    unsigned long long *full = bar + 2, *empty = bar + 4;
    const int tid = threadIdx.x;
    // digit-like operands in [-64, 64] from a hash of the byte index
    for (int i = tid; i < (A_BYTES + B_BYTES) / 4; i += 128) {
        unsigned h = (unsigned)i * 2654435761u + 0x9E3779B9u * (blockIdx.x + 1), w = 0;
        h ^= h >> 15;
        h *= 2246822519u;
        h ^= h >> 13;
#pragma unroll
        for (int b = 0; b < 4; ++b) w |= (unsigned)(unsigned char)(signed char)((int)((h >> (8 * b)) % 129u) - 64) << (8 * b);
        reinterpret_cast<unsigned *>(sm)[i] = w;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (tid == 0) {
        for (int q = 0; q < 5; ++q) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(i8_saddr(q == 0 ? bar : bar + 1 + q)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < 32) {
        if constexpr (PAIR)
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(i8_saddr(tslot)) : "memory");
        else
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(i8_saddr(tslot)) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    if constexpr (PAIR) i8_cluster_sync(); else __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tslot;
    unsigned rank = 0;
    if constexpr (PAIR) asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    if (tid == 0 && rank == 0) {
        const unsigned long long dA = i8_desc(sm), dB = i8_desc(sm + A_BYTES);
        if constexpr (HS) {
            int st = 0;
            unsigned ph = 0;
            for (int it = 0; it < iters; it += 2) {
                if (!i8_wait(full + st, ph)) {
                    atomicOr(status, 2);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                i8_kstep<N, PAIR, 0, 0>(tmem, dA, dB, 0);
                i8_kstep<N, PAIR, 0, 0>(tmem, dA, dB, 1);
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(i8_saddr(empty + st))
                             : "memory");
                if (++st == 2) {
                    st = 0;
                    ph ^= 1;
                }
            }
        } else {
            for (int it = 0; it < iters; ++it) i8_kstep<N, PAIR, 0, 0>(tmem, dA, dB, it & 1);
        }
        if constexpr (PAIR)
            asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
                             i8_saddr(bar)),
                         "h"((unsigned short)3)
                         : "memory");
        else
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(i8_saddr(bar))
                         : "memory");
    } else if (HS && !PAIR && tid == 32) {  // re-arms the ring as the MMAs release its stages
        int st = 0;
        unsigned ph = 0;
        for (int it = 0; it < iters; it += 2) {
            if (!i8_wait(empty + st, ph ^ 1)) {
                atomicOr(status, 4);
                break;
            }
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(i8_saddr(full + st)) : "memory");
            if (++st == 2) {
                st = 0;
                ph ^= 1;
            }
        }
    }
    // every CTA waits for its completion arrival (the pair's odd CTA gets the multicast one); tensor
    // memory is freed only after it, or after the bounded wait ran out
    if (tid == 0 && !i8_wait(bar, 0)) atomicOr(status, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    if constexpr (PAIR) i8_cluster_sync(); else __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid < 32) {
        if constexpr (PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
        else
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
    }
    if constexpr (PAIR) i8_cluster_sync();
}

}  // namespace probe
}  // namespace trpdrv

using namespace trpdrv;

static int launch_probe(int kind, int grid, int iters, double *sink, double *flops, cudaStream_t st)
{
    const double warps = (double)grid * (probe::NTHREAD / 32);
    const double per_iter = probe::NACC;
    double mma_flops = 0.0;
    switch (kind) {
    case 0:
        probe::probe_kernel<0><<<grid, probe::NTHREAD, 0, st>>>(iters, sink);
        mma_flops = 2.0 * 8 * 8 * 4;
        break;
    case 1:
        probe::probe_kernel<1><<<grid, probe::NTHREAD, 0, st>>>(iters, sink);
        mma_flops = 2.0 * 16 * 8 * 4;
        break;
    case 2:
        probe::probe_kernel<2><<<grid, probe::NTHREAD, 0, st>>>(iters, sink);
        mma_flops = 2.0 * 16 * 8 * 8;
        break;
    case 3:
        probe::probe_kernel<3><<<grid, probe::NTHREAD, 0, st>>>(iters, sink);
        mma_flops = 2.0 * 16 * 8 * 16;
        break;
    case 4:
        probe::probe_kernel<4><<<grid, probe::NTHREAD, 0, st>>>(iters, sink);
        mma_flops = 2.0 * 4 * 32;  // 4 DFMA per accumulator per lane
        break;
    default:
        return (int)cudaErrorInvalidValue;
    }
    if (flops) *flops = warps * iters * per_iter * mma_flops;
    return (int)cudaGetLastError();
}

// FP64 issue rate of `device` (-1 = current): kind 0 = DMMA m8n8k4, 1 = m16n8k4, 2 = m16n8k8,
// 3 = m16n8k16, 4 = scalar DFMA.  The loop grows until one launch takes >= 50 ms; writes TFLOP/s.
// Returns 0, or a CUDA error code.
extern "C" int trpdrv_probe_fp64_peak(int device, int kind, double *tflops)
{
    if (!tflops || kind < 0 || kind > 4) return (int)cudaErrorInvalidValue;
    cudaError_t e = cudaSuccess;
    if (device >= 0 && (e = cudaSetDevice(device)) != cudaSuccess) return (int)e;
    int dev = 0, nsm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return (int)e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return (int)e;
    const int grid = nsm * 4;
    double *sink = nullptr;
    if ((e = cudaMalloc((void **)&sink, sizeof(double) * (size_t)grid * probe::NTHREAD)) != cudaSuccess) return (int)e;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double flops = 0.0;
    int iters = 256, rc = 0;
    float ms = 0.0f;
    for (int attempt = 0; attempt < 12 && rc == 0; ++attempt) {
        rc = launch_probe(kind, grid, iters, sink, &flops, nullptr);  // warm-up
        if (rc) break;
        cudaEventRecord(e0, nullptr);
        rc = launch_probe(kind, grid, iters, sink, &flops, nullptr);
        if (rc) break;
        cudaEventRecord(e1, nullptr);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) {
            rc = (int)e;
            break;
        }
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms >= 50.0f) break;
        iters *= 2;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (rc) return rc;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return 0;
}

template <int N, bool PAIR, bool HS>
static int launch_int8_probe(int grid, int iters, int *status)
{
    const void *fn = (const void *)probe::int8_probe_kernel<N, PAIR, HS>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, probe::I8_SMEM);
    if (e != cudaSuccess) return (int)e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = probe::I8_SMEM;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = PAIR ? 2 : 1;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, probe::int8_probe_kernel<N, PAIR, HS>, iters, status);
    return (int)(e != cudaSuccess ? e : cudaGetLastError());
}

template <int N>
static int launch_int8_form(int flags, int grid, int iters, int *status)
{
    if (flags == 1) return launch_int8_probe<N, true, false>(grid, iters, status);
    if (flags == 2) return launch_int8_probe<N, false, true>(grid, iters, status);
    return launch_int8_probe<N, false, false>(grid, iters, status);
}

// int8 tensor-pipe rate of `device` (-1 = current) for tcgen05.mma.kind::i8 with K = 32 and N = 64,
// 128 or 256 over shared-memory operands: flags 0 = one issuing thread per SM, M = 128; 1 = CTA pairs
// (cta_group::2, M = 256, one issuing thread per pair); 2 = one SM per issuer behind the two-stage
// stage handshake of the contraction kernel.  The loop grows until one launch takes >= 20 ms; writes
// tera-operations per second (2 per multiply-add).  Returns 0, a CUDA error code, or -1 if a
// completion wait ran out.
extern "C" int trpdrv_probe_int8_rate(int device, int n, int flags, double *tops)
{
    if (!tops || (n != 64 && n != 128 && n != 256) || flags < 0 || flags > 2) return (int)cudaErrorInvalidValue;
    cudaError_t e = cudaSuccess;
    if (device >= 0 && (e = cudaSetDevice(device)) != cudaSuccess) return (int)e;
    int dev = 0, nsm = 0, major = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return (int)e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return (int)e;
    if ((e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev)) != cudaSuccess) return (int)e;
    if (major != 10) return (int)cudaErrorInvalidDevice;
    const int grid = nsm & ~1;  // pairs need an even grid; one CTA per SM either way
    int *status = nullptr;
    if ((e = cudaMalloc((void **)&status, sizeof(int))) != cudaSuccess) return (int)e;
    cudaMemset(status, 0, sizeof(int));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto launch = [&](int iters) {
        return n == 64 ? launch_int8_form<64>(flags, grid, iters, status)
             : n == 128 ? launch_int8_form<128>(flags, grid, iters, status) : launch_int8_form<256>(flags, grid, iters, status);
    };
    int iters = 256, rc = 0;
    float ms = 0.0f;
    for (int attempt = 0; attempt < 10 && rc == 0; ++attempt) {
        rc = launch(iters);  // warm-up
        if (rc) break;
        cudaEventRecord(e0, nullptr);
        rc = launch(iters);
        if (rc) break;
        cudaEventRecord(e1, nullptr);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) {
            rc = (int)e;
            break;
        }
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms >= 20.0f) break;
        iters *= 2;
    }
    int h_status = 0;
    if (!rc && (e = cudaMemcpy(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) rc = (int)e;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(status);
    if (rc) return rc;
    if (h_status) return -1;
    // every SM's tensor pipe does iters x 28 products x 128 rows x N x 32 multiply-adds per launch
    *tops = 2.0 * grid * (double)iters * 28.0 * 128.0 * n * 32.0 / (ms * 1e-3) / 1e12;
    return 0;
}

// The device's int8 rate for the single-SM form (flags 0).
extern "C" int trpdrv_probe_int8_peak(int device, int n, double *tops)
{
    return trpdrv_probe_int8_rate(device, n, 0, tops);
}
