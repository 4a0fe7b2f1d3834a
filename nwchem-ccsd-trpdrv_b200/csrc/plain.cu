// Plain per-triple path (sm_100a, FP64 DMMA): the reference body's structure on the GPU.
//
//  plain_gemm_kernel: one grouped launch computes all eight f of one triple into f[8][nvir][nvir]
//    (the 16 DGEMMs of omp/ccsd_trpdrv_omp_cbody.c:70-117: each f is its K=nvir product followed by
//    its K=nocc product, here one contraction over the concatenated index with the occupied A
//    operand pre-negated).  64x64 output tile per CTA, 4 warps of 32x32, cp.async 3-stage pipeline.
//  tengy_kernel: the (b,c) reduction of omp/ccsd_tengy_c99.c:5-119 over f in HBM, one CTA per
//    32-wide tile pair; the last CTA to finish sums the per-CTA partials in a fixed order.

#include "device_common.cuh"
#include "launch.h"
#include "tengy_tile.cuh"

namespace trpdrv {
namespace plain {

constexpr int BM = 64;           // output tile (rows b, cols c)
constexpr int DK = 8;
constexpr int STAGES = 3;
constexpr int NTHREAD = 128;
constexpr int PK = BM + 8;       // K-major pitch (== 8 mod 16)
constexpr int QX = DK + 4;       // X-major pitch
constexpr int APANEL = DK * PK;
constexpr int BPANEL = (DK * PK > BM * QX) ? DK * PK : BM * QX;
constexpr int STAGE = APANEL + BPANEL;
constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE * sizeof(double);

struct Src {
    const double *a, *b;
    int lda, ldb, bk, klim;
};

template <int VEC>
__device__ __forceinline__ void load_stage(double *stage, const Src &s, int r0, int c0, int kk0, int nvir,
                                           int tid)
{
    // A: K-major panel, rows r0.., element (r, kk) at a[r + kk*lda]
    constexpr int ACP = BM * DK / VEC;
#pragma unroll
    for (int u = 0; u < ACP / NTHREAD; ++u) {
        const int q = tid + u * NTHREAD;
        const int kk = q / (BM / VEC), r = (q % (BM / VEC)) * VEC;
        const bool ok = (r0 + r < nvir) && (kk0 + kk < s.klim);
        const double *src = ok ? s.a + (r0 + r) + (size_t)(kk0 + kk) * s.lda : s.a;
        double *dst = stage + kk * PK + r;
        if (VEC == 2) cp_async_16(dst, src, ok); else cp_async_8(dst, src, ok);
    }
    double *bst = stage + APANEL;
    constexpr int BCP = BM * DK / VEC;
#pragma unroll
    for (int u = 0; u < BCP / NTHREAD; ++u) {
        const int q = tid + u * NTHREAD;
        if (s.bk) {  // B(kk, c) = b[c + kk*ldb]
            const int kk = q / (BM / VEC), c = (q % (BM / VEC)) * VEC;
            const bool ok = (c0 + c < nvir) && (kk0 + kk < s.klim);
            const double *src = ok ? s.b + (c0 + c) + (size_t)(kk0 + kk) * s.ldb : s.b;
            double *dst = bst + kk * PK + c;
            if (VEC == 2) cp_async_16(dst, src, ok); else cp_async_8(dst, src, ok);
        } else {     // B(kk, c) = b[kk + c*ldb]
            const int c = q / (DK / VEC), d = (q % (DK / VEC)) * VEC;
            const bool ok = (c0 + c < nvir) && (kk0 + d < s.klim);
            const double *src = ok ? s.b + (kk0 + d) + (size_t)(c0 + c) * s.ldb : s.b;
            double *dst = bst + c * QX + d;
            if (VEC == 2) cp_async_16(dst, src, ok); else cp_async_8(dst, src, ok);
        }
    }
}

template <int VEC>
__global__ void __launch_bounds__(NTHREAD)
plain_gemm_kernel(const trpdrv_plain_args args)
{
    extern __shared__ __align__(16) double smem[];
    const int x = blockIdx.z;
    const int nvir = args.nvir, nocc = args.nocc;
    const int r0 = blockIdx.x * BM, c0 = blockIdx.y * BM;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    const int g = lane >> 2, t = lane & 3;

    Src ph[2];
    ph[0].a = args.a1[x];
    ph[0].lda = nvir;
    ph[0].b = args.b1[x];
    ph[0].ldb = nvir;
    ph[0].bk = args.b1_nt[x];
    ph[0].klim = nvir;
    ph[1].a = args.a2[x];
    ph[1].lda = nvir;
    ph[1].b = args.b2[x];
    ph[1].ldb = nocc;
    ph[1].bk = 0;
    ph[1].klim = nocc;
    const int nV = (nvir + DK - 1) / DK, nO = (nocc + DK - 1) / DK, nch = nV + nO;

    double acc[2][4][4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[mi][ni][e] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < nch) {
            const int p = s < nV ? 0 : 1;
            load_stage<VEC>(smem + s * STAGE, ph[p], r0, c0, (p ? s - nV : s) * DK, nvir, tid);
        }
        cp_async_commit();
    }
    for (int ch = 0; ch < nch; ++ch) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        const int nx = ch + STAGES - 1;
        if (nx < nch) {
            const int p = nx < nV ? 0 : 1;
            load_stage<VEC>(smem + (nx % STAGES) * STAGE, ph[p], r0, c0, (p ? nx - nV : nx) * DK, nvir, tid);
        }
        cp_async_commit();
        const double *As = smem + (ch % STAGES) * STAGE;
        const double *Bs = As + APANEL;
        const bool bK = (ch < nV) && ph[0].bk;
#pragma unroll
        for (int ks = 0; ks < DK / 4; ++ks) {
            const int kk = ks * 4 + t;
            double a[2][2], b[4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                a[mi][0] = As[kk * PK + wm + mi * 16 + g];
                a[mi][1] = As[kk * PK + wm + mi * 16 + g + 8];
            }
            if (bK) {
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) b[ni] = Bs[kk * PK + wn + ni * 8 + g];
            } else {
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) b[ni] = Bs[(wn + ni * 8 + g) * QX + kk];
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], a[mi][0], a[mi][1], b[ni]);
        }
    }
    cp_async_wait<0>();

    double *f = args.f + (size_t)x * nvir * nvir;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            const int r = r0 + wm + mi * 16 + g, c = c0 + wn + ni * 8 + 2 * t;
            if (r < nvir && c < nvir) f[r + (size_t)c * nvir] = acc[mi][ni][0];
            if (r < nvir && c + 1 < nvir) f[r + (size_t)(c + 1) * nvir] = acc[mi][ni][1];
            if (r + 8 < nvir && c < nvir) f[r + 8 + (size_t)c * nvir] = acc[mi][ni][2];
            if (r + 8 < nvir && c + 1 < nvir) f[r + 8 + (size_t)(c + 1) * nvir] = acc[mi][ni][3];
        }
}

// ------------------------------------------------------------------------------------------------
constexpr int TNTHREAD = 512;
constexpr size_t TSMEM_BYTES = (size_t)16 * TPTILE * sizeof(double);

__global__ void __launch_bounds__(TNTHREAD, 1)
tengy_kernel(const trpdrv_tengy_args args)
{
    extern __shared__ __align__(16) double park[];
    __shared__ double red[4 * (TNTHREAD / 32)];
    __shared__ int s_last;
    const int nvir = args.nvir;
    const int nb = (nvir + TT - 1) / TT;
    const int tid = threadIdx.x;

    int B = 0, rem = blockIdx.x;
    while (B < nb && rem >= nb - B) {
        rem -= nb - B;
        ++B;
    }
    const int C = B + rem;
    const int b0 = B * TT, c0 = C * TT;
    const bool diag = (B == C);
    const size_t lnvv = (size_t)nvir * nvir;

    // stage f(B,C) (o = 0) and f(C,B) (o = 1) tiles of all eight f; out-of-range entries are zero
    const int ntiles = diag ? 8 : 16;
    for (int idx = tid; idx < ntiles * TT * TT; idx += TNTHREAD) {
        const int tile = idx >> 10, q = (idx >> 5) & 31, r = idx & 31;
        const int o = tile >> 3, xf = tile & 7;
        const int row = (o ? c0 : b0) + r, col = (o ? b0 : c0) + q;
        double v = 0.0;
        if (row < nvir && col < nvir) v = args.f[(size_t)xf * lnvv + row + (size_t)col * nvir];
        park[tile * TPTILE + r * TPP + q] = v;
    }
    __syncthreads();

    TengyVecs v;
    v.eorb = args.eorb;
    v.dintc1 = args.dintc1;
    v.dintx1 = args.dintx1;
    v.t1v1 = args.t1v1;
    v.dintc2 = args.dintc2;
    v.dintx2 = args.dintx2;
    v.t1v2 = args.t1v2;
    v.voff = args.ncor + args.nocc;
    v.nvir = nvir;
    if (args.use_eaijk)
        v.eaijk = args.eaijk;
    else  // omp/ccsd_trpdrv_omp_cbody.c:126
        v.eaijk = args.eorb[args.a - 1] - (args.eorb[args.ncor + args.i - 1] + args.eorb[args.ncor + args.j - 1] +
                                            args.eorb[args.ncor + args.k - 1]);
    TengySums su = {0.0, 0.0, 0.0, 0.0};
    tengy_tile_pair(park, b0, c0, diag, v, tid, TNTHREAD, su);
    const TengySums tot = block_sum4(su, red);

    if (tid == 0) {
        double *bp = args.block_partial + 4 * blockIdx.x;
        bp[0] = tot.e4i;
        bp[1] = tot.e5i;
        bp[2] = tot.e4k;
        bp[3] = tot.e5k;
        __threadfence();
        const unsigned prev = atomicAdd(args.counter, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (s_last && tid == 0) {
        __threadfence();
        double s4i = 0.0, s5i = 0.0, s4k = 0.0, s5k = 0.0;
        for (unsigned blk = 0; blk < gridDim.x; ++blk) {
            const double *bp = args.block_partial + 4 * blk;
            s4i += __ldcg(bp + 0);
            s5i += __ldcg(bp + 1);
            s4k += __ldcg(bp + 2);
            s5k += __ldcg(bp + 3);
        }
        args.out4[0] = s4i;
        args.out4[1] = s5i;
        args.out4[2] = s4k;
        args.out4[3] = s5k;
        *args.counter = 0u;
    }
}

}  // namespace plain
}  // namespace trpdrv

using namespace trpdrv;

extern "C" int trpdrv_launch_plain_gemm(const trpdrv_plain_args *args, int vec2, void *stream)
{
    const int nbt = (args->nvir + plain::BM - 1) / plain::BM;
    dim3 grid(nbt, nbt, 8);
    cudaStream_t st = (cudaStream_t)stream;
    if (vec2)
        plain::plain_gemm_kernel<2><<<grid, plain::NTHREAD, plain::SMEM_BYTES, st>>>(*args);
    else
        plain::plain_gemm_kernel<1><<<grid, plain::NTHREAD, plain::SMEM_BYTES, st>>>(*args);
    return (int)cudaGetLastError();
}

extern "C" size_t trpdrv_tengy_smem_bytes(void) { return plain::TSMEM_BYTES; }

extern "C" int trpdrv_launch_tengy(const trpdrv_tengy_args *args, void *stream)
{
    const int nb = (args->nvir + TT - 1) / TT;
    const int npairs = nb * (nb + 1) / 2;
    plain::tengy_kernel<<<npairs, plain::TNTHREAD, plain::TSMEM_BYTES, (cudaStream_t)stream>>>(*args);
    return (int)cudaGetLastError();
}

extern "C" int trpdrv_plain_init(void)
{
    cudaError_t e = cudaFuncSetAttribute(plain::plain_gemm_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)plain::SMEM_BYTES);
    if (e != cudaSuccess) return (int)e;
    e = cudaFuncSetAttribute(plain::plain_gemm_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)plain::SMEM_BYTES);
    if (e != cudaSuccess) return (int)e;
    return (int)cudaFuncSetAttribute(plain::tengy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)plain::TSMEM_BYTES);
}
