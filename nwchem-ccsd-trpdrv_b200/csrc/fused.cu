// Fused persistent triples kernel (sm_100a, FP64 DMMA).
//
// One launch processes every work item of a plan.  A work item is (triple (i,j,k), tile pair
// {B,C}) with B <= C over 32-wide blocks of the virtual index.  For its item a CTA computes, for all
// eight intermediates of omp/ccsd_trpdrv_omp_cbody.c:70-117, the 32x32 tiles f(B,C) and f(C,B)
// (16 tiles, one per warp), parks them in shared memory and evaluates the tengy terms
// (omp/ccsd_tengy_c99.c:58-111) of every (b,c) in BxC and CxB directly from there, so f never
// reaches HBM.  The per-item energies go to a slot array and are reduced in a fixed order by
// reduce.cu (deterministic; no floating-point atomics).
//
// Each f is one contraction over the concatenated index d = [virtual | occupied]:
//   f1n = [Jia | -Tia] [Tkj^T ; Kkj]   f2n = [Kia | -Xia] [Tkj^T ; Kkj]
//   f3n = [Jia | -Tia] [Tkj   ; Jkj]   f4n = [Kia | -Xia] [Tkj   ; Jkj]
//   f1t = [Jka | -Tka] [Tij^T ; Kij]   f2t = [Kka | -Xka] [Tij^T ; Kij]
//   f3t = [Jka | -Tka] [Tij   ; Jij]   f4t = [Kka | -Xka] [Tij   ; Jij]
// (the negated occupied operands are stored negated on the device, so every MMA accumulates with +1).
// Per item and chunk of DK contraction indices the CTA stages 16 panels (32 x DK) with cp.async:
// A-rows {J,K} x {B,C} and B-columns {1,3} x {C,B} for each of the n and t families; each panel
// feeds two warps.  Diagonal items (B == C) need only half of the panels and warps.
//
// Work distribution: an atomic ticket (one 64-bit atomicAdd per item); no CTA ever waits on another.

#include "device_common.cuh"
#include "launch.h"
#include "tengy_tile.cuh"

namespace trpdrv {
namespace fused {

constexpr int T = TRPDRV_TILE;   // 32
constexpr int DK = 8;            // contraction chunk per pipeline stage
constexpr int STAGES = 3;
constexpr int NWARP = 16;
constexpr int NTHREAD = NWARP * 32;
constexpr int PK = T + 8;        // K-major panel pitch (doubles); == 8 mod 16 -> conflict-free frags
constexpr int QX = DK + 4;       // X-major panel pitch
constexpr int PANEL = (DK * PK > T * QX) ? DK * PK : T * QX;
constexpr int NPANEL = 16;
constexpr int STAGE = NPANEL * PANEL;
constexpr int PP = T + 1;        // parked tile pitch
constexpr int PTILE = T * PP;
constexpr int PARK = 16 * PTILE;
constexpr int PIPE = STAGES * STAGE;
constexpr int MAIN = PIPE > PARK ? PIPE : PARK;
constexpr size_t SMEM_BYTES = (size_t)MAIN * sizeof(double);

static_assert(T == TT && PP == TPP, "park layout must match tengy_tile.cuh");
static_assert(DK % 4 == 0, "DK must be a multiple of the MMA k (4)");

struct PanelInfo {
    const double *base;  // element (first row or column of the panel, contraction index 0)
    int ld;              // leading dimension of the source matrix
    int rem;             // rows (K-major) / columns (X-major) of the panel that lie inside nvir
    int kmajor;          // 1: contraction index strided (rows contiguous); 0: contraction contiguous
    int pad;
};

struct ItemCtx {
    PanelInfo tbl[2][NPANEL];  // [phase 0 = virtual, 1 = occupied][panel]
    const double *eorb, *dintc1, *dintx1, *t1v1, *dintc2, *dintx2, *t1v2;
    double *out;
    double eaijk;
    int ncor, nocc, nvir, b0, c0, diag, nV, nO, valid;
};

template <int VEC>
__device__ __forceinline__ void load_stage(double *stage, const ItemCtx &cx, int ch, int tid)
{
    const int ph = ch < cx.nV ? 0 : 1;
    const int kk0 = (ph ? ch - cx.nV : ch) * DK;
    const int klim = ph ? cx.nocc : cx.nvir;
    constexpr int CPP = T * DK / VEC;        // copies per panel
    constexpr int ITER = NPANEL * CPP / NTHREAD;
    static_assert(NPANEL * CPP % NTHREAD == 0, "copies must split evenly over the CTA");
#pragma unroll
    for (int u = 0; u < ITER; ++u) {
        const int id = tid + u * NTHREAD;
        const int p = id / CPP;
        const int q = id % CPP;
        if (cx.diag && (p & 1)) continue;
        const PanelInfo &pi = cx.tbl[ph][p];
        double *dst = stage + p * PANEL;
        const double *src;
        bool ok;
        if (pi.kmajor) {
            const int kk = q / (T / VEC), r = (q % (T / VEC)) * VEC;
            ok = (r < pi.rem) && (kk0 + kk < klim);
            src = pi.base + r + (size_t)(kk0 + kk) * pi.ld;
            dst += kk * PK + r;
        } else {
            const int cc = q / (DK / VEC), d = (q % (DK / VEC)) * VEC;
            ok = (cc < pi.rem) && (kk0 + d < klim);
            src = pi.base + (kk0 + d) + (size_t)cc * pi.ld;
            dst += cc * QX + d;
        }
        if (!ok) src = cx.eorb;  // mapped address; zero-fill reads nothing
        if (VEC == 2)
            cp_async_16(dst, src, ok);
        else
            cp_async_8(dst, src, ok);
    }
}

__device__ __forceinline__ void compute_stage(const double *stage, int pa, int pb, bool bK, int lane,
                                              double (&acc)[2][4][4])
{
    const int g = lane >> 2, t = lane & 3;
    const double *As = stage + pa * PANEL;
    const double *Bs = stage + pb * PANEL;
#pragma unroll
    for (int ks = 0; ks < DK / 4; ++ks) {
        const int kk = ks * 4 + t;
        double a[2][2], b[4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
            a[mi][0] = As[kk * PK + mi * 16 + g];
            a[mi][1] = As[kk * PK + mi * 16 + g + 8];
        }
        if (bK) {
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) b[ni] = Bs[kk * PK + ni * 8 + g];
        } else {
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) b[ni] = Bs[(ni * 8 + g) * QX + kk];
        }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], a[mi][0], a[mi][1], b[ni]);
    }
}

// Fills the item context (warp 0 only).  Returns nothing; sets cx.valid = 0 and *status on a
// malformed queue entry (the item is then skipped with zero energies).
__device__ __forceinline__ void setup_item(const trpdrv_dev_system *__restrict__ sys, int nsys,
                                           long long item, ItemCtx &cx, int *status, int lane)
{
    int s = 0;
    while (s + 1 < nsys && item >= sys[s + 1].item_begin) ++s;
    const trpdrv_dev_system &S = sys[s];
    const long long local = item - S.item_begin;
    const long long tt = local / S.npairs;
    const int p = (int)(local - tt * S.npairs);
    int B = 0, rem = p;
    while (B < S.nb && rem >= S.nb - B) {
        rem -= S.nb - B;
        ++B;
    }
    const int C = B + rem;
    const int O = S.nocc, V = S.nvir;
    int packed = 0;
    bool ok = (tt >= 0) && (tt < S.ntriples) && (B < S.nb) && (C < S.nb);
    if (ok) packed = S.triples[tt];
    const int i = packed & 1023, j = (packed >> 10) & 1023, k = (packed >> 20) & 1023;
    ok = ok && (i < O) && (j < O) && (k < O) && (k <= i);
    if (!ok) {
        if (lane == 0) {
            atomicExch(status, 1);
            cx.valid = 0;
            const bool in_range = local >= 0 && local < S.ntriples * (long long)S.npairs;
            cx.out = in_range ? S.partial + 4 * local : nullptr;
        }
        return;
    }
    const size_t lnvv = (size_t)V * V, lnov = (size_t)O * V;
    const size_t jo = (size_t)j * O;
    const int B0 = B * T, C0 = C * T;

    // panel table: lane -> (phase, panel)
    {
        const int ph = lane >> 4, pnl = lane & 15, fam = pnl >> 3, q = pnl & 7;
        const double *Aj, *Ak, *B1, *B3;
        if (fam == 0) {
            Aj = ph ? S.ntov + (size_t)i * lnov : S.jvv + (size_t)i * lnvv;
            Ak = ph ? S.nxov + (size_t)i * lnov : S.kvv + (size_t)i * lnvv;
            B1 = ph ? S.kov + (jo + k) * lnov : S.t2 + (jo + k) * lnvv;
            B3 = ph ? S.jov + (jo + k) * lnov : S.t2 + (jo + k) * lnvv;
        } else {
            Aj = ph ? S.ntov + (size_t)k * lnov : S.jvv + (size_t)k * lnvv;
            Ak = ph ? S.nxov + (size_t)k * lnov : S.kvv + (size_t)k * lnvv;
            B1 = ph ? S.kov + (jo + i) * lnov : S.t2 + (jo + i) * lnvv;
            B3 = ph ? S.jov + (jo + i) * lnov : S.t2 + (jo + i) * lnvv;
        }
        PanelInfo pi;
        pi.pad = 0;
        if (q < 4) {
            const int off = (q & 1) ? C0 : B0;  // A rows: B for orientation (B,C), C for (C,B)
            pi.base = ((q >> 1) ? Ak : Aj) + off;
            pi.ld = V;
            pi.rem = V - off;
            pi.kmajor = 1;
        } else {
            const int off = (q & 1) ? B0 : C0;  // B columns: C for (B,C), B for (C,B)
            pi.rem = V - off;
            if (q < 6) {                        // [T^T ; K]: T(c,d) rows contiguous, K(m,c) m contiguous
                if (ph == 0) {
                    pi.base = B1 + off;
                    pi.ld = V;
                    pi.kmajor = 1;
                } else {
                    pi.base = B1 + (size_t)off * O;
                    pi.ld = O;
                    pi.kmajor = 0;
                }
            } else {                            // [T ; J]: contraction index contiguous in both
                pi.base = B3 + (size_t)off * (ph ? O : V);
                pi.ld = ph ? O : V;
                pi.kmajor = 0;
            }
        }
        cx.tbl[ph][pnl] = pi;
    }
    if (lane == 0) {
        cx.eorb = S.eorb;
        cx.dintc1 = S.dintc + (size_t)i * V;
        cx.dintx1 = S.dintx + (size_t)i * V;
        cx.t1v1 = S.t1v + (size_t)i * V;
        cx.dintc2 = S.dintc + (size_t)k * V;
        cx.dintx2 = S.dintx + (size_t)k * V;
        cx.t1v2 = S.t1v + (size_t)k * V;
        cx.out = S.partial + 4 * local;
        // omp/ccsd_trpdrv_omp_cbody.c:126 (a is 1-based, i/j/k here 0-based)
        cx.eaijk = S.eorb[S.a - 1] - (S.eorb[S.ncor + i] + S.eorb[S.ncor + j] + S.eorb[S.ncor + k]);
        cx.ncor = S.ncor;
        cx.nocc = O;
        cx.nvir = V;
        cx.b0 = B0;
        cx.c0 = C0;
        cx.diag = (B == C);
        cx.nV = (V + DK - 1) / DK;
        cx.nO = (O + DK - 1) / DK;
        cx.valid = 1;
    }
}

template <int VEC>
__global__ void __launch_bounds__(NTHREAD, 1)
fused_kernel(const trpdrv_dev_system *__restrict__ sys, int nsys, long long total,
             unsigned long long *counter, int *status)
{
    extern __shared__ __align__(16) double smem[];
    __shared__ ItemCtx cx;
    __shared__ double red[4 * NWARP];
    __shared__ long long s_item;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int fam = warp >> 3, x = (warp >> 1) & 3, o = warp & 1;
    const int pa = fam * 8 + ((x & 1) ? 2 : 0) + o;
    const int pb = fam * 8 + 4 + ((x >= 2) ? 2 : 0) + o;
    const int g = lane >> 2, t4 = lane & 3;

    for (;;) {
        if (tid == 0) s_item = (long long)atomicAdd(counter, 1ULL);
        __syncthreads();
        const long long item = s_item;
        if (item >= total) break;
        if (warp == 0) setup_item(sys, nsys, item, cx, status, lane);
        __syncthreads();
        if (!cx.valid) {
            if (tid < 4 && cx.out) cx.out[tid] = 0.0;
            continue;
        }

        const int nch = cx.nV + cx.nO;
        const bool diag = cx.diag != 0;
        const bool active = !(diag && o);
        double acc[2][4][4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[mi][ni][e] = 0.0;

#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s) {
            if (s < nch) load_stage<VEC>(smem + s * STAGE, cx, s, tid);
            cp_async_commit();
        }
        for (int ch = 0; ch < nch; ++ch) {
            cp_async_wait<STAGES - 2>();
            __syncthreads();
            const int nx = ch + STAGES - 1;
            if (nx < nch) load_stage<VEC>(smem + (nx % STAGES) * STAGE, cx, nx, tid);
            cp_async_commit();
            if (active) {
                const bool bK = (ch < cx.nV) && (x < 2);
                compute_stage(smem + (ch % STAGES) * STAGE, pa, pb, bK, lane, acc);
            }
        }
        cp_async_wait<0>();
        __syncthreads();

        // park f tiles: tile index = orientation*8 + f index (f1n f2n f3n f4n f1t f2t f3t f4t)
        if (active) {
            double *tile = smem + (o * 8 + fam * 4 + x) * PTILE;
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) {
                    const int r = mi * 16 + g, c = ni * 8 + 2 * t4;
                    tile[r * PP + c] = acc[mi][ni][0];
                    tile[r * PP + c + 1] = acc[mi][ni][1];
                    tile[(r + 8) * PP + c] = acc[mi][ni][2];
                    tile[(r + 8) * PP + c + 1] = acc[mi][ni][3];
                }
        }
        __syncthreads();

        // tengy epilogue over BxC and CxB (tengy_tile.cuh)
        TengySums su = {0.0, 0.0, 0.0, 0.0};
        {
            TengyVecs v;
            v.eorb = cx.eorb;
            v.dintc1 = cx.dintc1;
            v.dintx1 = cx.dintx1;
            v.t1v1 = cx.t1v1;
            v.dintc2 = cx.dintc2;
            v.dintx2 = cx.dintx2;
            v.t1v2 = cx.t1v2;
            v.eaijk = cx.eaijk;
            v.voff = cx.ncor + cx.nocc;
            v.nvir = cx.nvir;
            tengy_tile_pair(smem, cx.b0, cx.c0, diag, v, tid, NTHREAD, su);
        }
        const TengySums tot = block_sum4(su, red);
        if (tid == 0) {
            double *out = cx.out;
            out[0] = tot.e4i;
            out[1] = tot.e5i;
            out[2] = tot.e4k;
            out[3] = tot.e5k;
        }
    }
}

}  // namespace fused
}  // namespace trpdrv

using namespace trpdrv;

extern "C" size_t trpdrv_fused_smem_bytes(void) { return fused::SMEM_BYTES; }
extern "C" int trpdrv_fused_threads(void) { return fused::NTHREAD; }

extern "C" int trpdrv_fused_max_ctas_per_sm(int *n)
{
    return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, fused::fused_kernel<2>, fused::NTHREAD,
                                                              fused::SMEM_BYTES);
}

extern "C" int trpdrv_launch_fused(const trpdrv_dev_system *d_sys, int nsys, int64_t total_items,
                                   unsigned long long *counter, int *status, int grid, int vec2,
                                   void *stream)
{
    if (grid <= 0 || total_items <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    if (vec2)
        fused::fused_kernel<2><<<grid, fused::NTHREAD, fused::SMEM_BYTES, st>>>(d_sys, nsys, total_items,
                                                                               counter, status);
    else
        fused::fused_kernel<1><<<grid, fused::NTHREAD, fused::SMEM_BYTES, st>>>(d_sys, nsys, total_items,
                                                                               counter, status);
    return (int)cudaGetLastError();
}

extern "C" int trpdrv_fused_init(void)
{
    cudaError_t e = cudaFuncSetAttribute(fused::fused_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fused::SMEM_BYTES);
    if (e != cudaSuccess) return (int)e;
    return (int)cudaFuncSetAttribute(fused::fused_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)fused::SMEM_BYTES);
}
