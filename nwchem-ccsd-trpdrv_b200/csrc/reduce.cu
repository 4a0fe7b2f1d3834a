// Deterministic energy reductions and small device utilities.
//
//  item_reduce_kernel:   per triple, the compensated sum of its tile-pair items (fixed order) -> rec[t][4]
//  system_reduce_kernel: per system, the compensated total of emp4i + [i != k] emp4k and of
//                        emp5i + [i != k] emp5k over the triples (the accumulation of
//                        omp/ccsd_trpdrv_omp_cbody.c:133-142), as a double-double (hi, lo) pair,
//                        built with error-free TwoSum in a fixed order.
//  negate_kernel:        dst = -src (the occupied A operands are stored negated).
//  gather_kernel:        a list of device-to-device copies in one launch (the drop-in entry points'
//                        registered inputs, gathered into their staging layout).

#include "device_common.cuh"
#include "launch.h"

namespace trpdrv {

__global__ void item_reduce_kernel(const double *__restrict__ partial, int npairs, long long ntriples,
                                   double *__restrict__ rec)
{
    const long long t = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= ntriples) return;
    const int nslot = npairs * TRPDRV_FUSED_SLOTS;
    const double *p = partial + 4 * t * (long long)nslot;
    // compensated per lane (error-free TwoSum, errors carried in lo), then the lanes' hi and lo sums
    double hi[4] = {0.0, 0.0, 0.0, 0.0}, lo[4] = {0.0, 0.0, 0.0, 0.0};
    for (int q = lane; q < nslot; q += 32) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            double s, e;
            two_sum(hi[c], p[4 * q + c], s, e);
            hi[c] = s;
            lo[c] += e;
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double h = warp_sum(hi[c]), l = warp_sum(lo[c]);
        if (lane == 0) rec[4 * t + c] = h + l;
    }
}

__device__ __forceinline__ void dd_add(double &hi, double &lo, double x)
{
    double s, e;
    two_sum(hi, x, s, e);
    hi = s;
    lo += e;
}

constexpr int RED_THREADS = 1024;

__global__ void __launch_bounds__(RED_THREADS)
system_reduce_kernel(const double *__restrict__ rec, const int32_t *__restrict__ triples, long long n, long long nt,
                     double *__restrict__ out)
{
    __shared__ double sh[4][RED_THREADS];
    double h4 = 0.0, l4 = 0.0, h5 = 0.0, l5 = 0.0;
    for (long long t = threadIdx.x; t < n; t += RED_THREADS) {
        const int packed = triples[t % nt];  // records are [a][triple]
        const int i = packed & 1023, k = (packed >> 20) & 1023;
        dd_add(h4, l4, rec[4 * t + 0]);
        dd_add(h5, l5, rec[4 * t + 1]);
        if (i != k) {
            dd_add(h4, l4, rec[4 * t + 2]);
            dd_add(h5, l5, rec[4 * t + 3]);
        }
    }
    sh[0][threadIdx.x] = h4;
    sh[1][threadIdx.x] = l4;
    sh[2][threadIdx.x] = h5;
    sh[3][threadIdx.x] = l5;
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            const int o = threadIdx.x + w;
            double s, e;
            two_sum(sh[0][threadIdx.x], sh[0][o], s, e);
            sh[0][threadIdx.x] = s;
            sh[1][threadIdx.x] += sh[1][o] + e;
            two_sum(sh[2][threadIdx.x], sh[2][o], s, e);
            sh[2][threadIdx.x] = s;
            sh[3][threadIdx.x] += sh[3][o] + e;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double s, e;
        two_sum(sh[0][0], sh[1][0], s, e);  // renormalise
        out[0] = s;
        out[1] = e;
        two_sum(sh[2][0], sh[3][0], s, e);
        out[2] = s;
        out[3] = e;
    }
}

__global__ void negate_kernel(const double *__restrict__ src, double *__restrict__ dst, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = -src[i];
}

// One row of the grid per segment; 16-byte copies when source and destination allow them.
__global__ void gather_kernel(const trpdrv_copy_list L)
{
    const int s = blockIdx.y;
    if (s >= L.n) return;
    const double *src = L.src[s];
    double *dst = L.dst[s];
    const long long n = L.len[s];
    const double sg = L.neg[s] ? -1.0 : 1.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15u) == 0) {
        const long long n2 = n >> 1;
        for (long long q = t0; q < n2; q += stride) {
            const double2 v = __ldg(reinterpret_cast<const double2 *>(src) + q);
            reinterpret_cast<double2 *>(dst)[q] = make_double2(sg * v.x, sg * v.y);
        }
        if ((n & 1) && t0 == 0) dst[n - 1] = sg * src[n - 1];
    } else {
        for (long long q = t0; q < n; q += stride) dst[q] = sg * src[q];
    }
}

}  // namespace trpdrv

using namespace trpdrv;

extern "C" int trpdrv_launch_gather(const trpdrv_copy_list *list, void *stream)
{
    if (!list || list->n <= 0) return 0;
    if (list->n > TRPDRV_COPY_LIST_MAX) return (int)cudaErrorInvalidValue;
    long long longest = 0;
    for (int s = 0; s < list->n; ++s) longest = list->len[s] > longest ? list->len[s] : longest;
    long long bx = (longest / 2 + 255) / 256;
    if (bx < 1) bx = 1;
    if (bx > 64) bx = 64;
    gather_kernel<<<dim3((unsigned)bx, (unsigned)list->n), 256, 0, (cudaStream_t)stream>>>(*list);
    return (int)cudaGetLastError();
}

extern "C" int trpdrv_launch_item_reduce(const trpdrv_dev_system *h_sys, void *stream)
{
    if (h_sys->ntriples <= 0) return 0;
    const int warps = 8;
    const long long blocks = (h_sys->ntriples + warps - 1) / warps;
    item_reduce_kernel<<<(unsigned)blocks, warps * 32, 0, (cudaStream_t)stream>>>(h_sys->partial, h_sys->npairs,
                                                                                 h_sys->ntriples, h_sys->rec);
    return (int)cudaGetLastError();
}

extern "C" int trpdrv_launch_system_reduce(const double *rec, const int32_t *triples, int64_t ntriples, int64_t nt,
                                           double *out, void *stream)
{
    if (nt <= 0) return 0;
    system_reduce_kernel<<<1, RED_THREADS, 0, (cudaStream_t)stream>>>(rec, triples, (long long)ntriples, (long long)nt,
                                                                     out);
    return (int)cudaGetLastError();
}

extern "C" int trpdrv_launch_negate(const double *src, double *dst, size_t n, void *stream)
{
    if (n == 0) return 0;
    size_t blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    negate_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(src, dst, n);
    return (int)cudaGetLastError();
}
