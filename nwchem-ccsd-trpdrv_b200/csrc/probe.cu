// FP64 issue-rate probe: the roofline denominator for the FP64 contraction kernels.
//
// A measurement tool, not part of the product: it is built into its own library,
// lib/libtrpdrv_probe.so, which only the benchmark loads.
//
// Every warp keeps NACC independent accumulator chains in registers and issues NACC MMAs (or DFMAs)
// per iteration with register operands only, so the measured rate is the FP64 tensor (or FMA) pipe
// throughput of the device, not a memory rate.  The accumulators are written out at the end so the
// work cannot be eliminated.

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
