// Fused persistent triples kernel (sm_100a, FP64 DMMA).
//
// One launch processes every work item of a plan.  A work item is (triple (i,j,k), tile pair
// {B,C}) with B <= C over 32-wide blocks of the virtual index.  The tengy sum of
// omp/ccsd_tengy_c99.c:58-111 over every (b,c) in BxC and CxB needs, at each position, all eight
// intermediates of omp/ccsd_trpdrv_omp_cbody.c:70-117 at (b,c) AND at (c,b).  Each warp owns a
// 16(b) x 8(c) sub-block of the pair and computes, for all eight f, both
//     f_x(b,c) = sum_d A_x(b,d) B_x(d,c)            (MMA with A rows b, B columns c)
//     g_x(b,c) = f_x(c,b) = sum_d B_x(d,b) A_x(c,d)  (the same MMA with the operand roles swapped)
// so f(b,c) and f(c,b) land in the same registers of the same thread and the energy terms are
// evaluated in registers: f never leaves the SM and the epilogue needs no shared memory.
//
// Each f is one contraction over the concatenated index d = [virtual | occupied]:
//   f1n = [Jia | -Tia] [Tkj^T ; Kkj]   f2n = [Kia | -Xia] [Tkj^T ; Kkj]
//   f3n = [Jia | -Tia] [Tkj   ; Jkj]   f4n = [Kia | -Xia] [Tkj   ; Jkj]
//   f1t = [Jka | -Tka] [Tij^T ; Kij]   f2t = [Kka | -Xka] [Tij^T ; Kij]
//   f3t = [Jka | -Tka] [Tij   ; Jij]   f4t = [Kka | -Xka] [Tij   ; Jij]
// (the negated occupied operands are stored negated on the device, so every MMA accumulates with +1).
// Per chunk of DK contraction indices the CTA stages 16 panels (32 x DK, padded) with cp.async:
// A rows {J,K} x {B,C} and B columns {1,3} x {C,B} for the n and t families.  The cp.async pipeline
// runs continuously across work items (the next items' chunks are in flight while the current item
// finishes), and work items come from an atomic ticket; no CTA ever waits on another.
//
// Per-warp energies go to partial[item][warp][4]; reduce.cu sums them in a fixed order.

#include "device_common.cuh"
#include "launch.h"

namespace trpdrv {
namespace fused {

constexpr int T = TRPDRV_TILE;     // 32
constexpr int DK = 8;              // contraction indices per pipeline stage
constexpr int STAGES = 4;
constexpr int NWARP = TRPDRV_FUSED_SLOTS;  // 8
constexpr int NTHREAD = NWARP * 32;
constexpr int QX = DK + 4;         // X-major panel pitch (contraction index contiguous)
constexpr int PANEL = T * QX;      // >= DK * PK for both K-major pitches below
constexpr int NPANEL = 16;
constexpr int STAGE = NPANEL * PANEL;
constexpr int RING = 8;            // item contexts in flight (>= STAGES + 2)
constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE * sizeof(double);

// K-major pitch: 40 (== 8 mod 16) for k4 fragments; 36 (== 4 mod 8) for the k-permuted k8 fragments.
template <int K> struct Pitch { static constexpr int PK = (K == 8) ? 36 : 40; };
static_assert(DK * 40 <= PANEL && DK * 36 <= PANEL, "panel slot too small");
static_assert(RING >= STAGES + 2, "context ring too small for the pipeline depth");

struct PanelInfo {
    const double *base;  // element (first row or column of the panel, contraction index 0)
    int ld;              // leading dimension of the source matrix
    int rem;             // rows (K-major) / columns (X-major) of the panel that lie inside nvir
    int kmajor;          // 1: rows contiguous, contraction index strided; 0: contraction contiguous
    int pad;
};

struct ItemCtx {
    PanelInfo tbl[2][NPANEL];  // [phase 0 = virtual, 1 = occupied][panel]
    const double *eorb, *dintc1, *dintx1, *t1v1, *dintc2, *dintx2, *t1v2;
    double *out;               // partial + item * NWARP * 4
    double eaijk;
    int ncor, nocc, nvir, b0, c0, diag, nV, nO, nch, state;  // state: 1 work, 0 skip (bad entry), -1 end
};

// ------------------------------------------------------------------------------------------------
// fragments.  el(P, kmajor, kk, x): element (contraction kk, row/column x) of a staged panel.
// k4: lane t holds contraction index ks*4+t.  k8: lane t holds logical k = t and t+4, stored at
// physical 2t and 2t+1 of the step (the same permutation for A and B keeps the product exact).
// ------------------------------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ double el(const double *P, bool km, int kk, int x)
{
    return km ? P[kk * Pitch<K>::PK + x] : P[x * QX + kk];
}

template <int K> struct Mma;

template <> struct Mma<4> {
    static constexpr int NA = 2, NB = 1;
    __device__ __forceinline__ static void ldA(double (&a)[2], const double *P, bool km, int ks, int x0, int g, int t)
    {
        const int kk = ks * 4 + t;
        a[0] = el<4>(P, km, kk, x0 + g);
        a[1] = el<4>(P, km, kk, x0 + g + 8);
    }
    __device__ __forceinline__ static void ldB(double (&b)[1], const double *P, bool km, int ks, int x0, int g, int t)
    {
        b[0] = el<4>(P, km, ks * 4 + t, x0 + g);
    }
    __device__ __forceinline__ static void mma(double (&d)[4], const double (&a)[2], const double (&b)[1])
    {
        dmma_16x8x4(d, a[0], a[1], b[0]);
    }
};

template <> struct Mma<8> {
    static constexpr int NA = 4, NB = 2;
    __device__ __forceinline__ static void ldA(double (&a)[4], const double *P, bool km, int ks, int x0, int g, int t)
    {
        const int kk = ks * 8 + 2 * t;
        if (km) {
            a[0] = P[kk * Pitch<8>::PK + x0 + g];
            a[1] = P[kk * Pitch<8>::PK + x0 + g + 8];
            a[2] = P[(kk + 1) * Pitch<8>::PK + x0 + g];
            a[3] = P[(kk + 1) * Pitch<8>::PK + x0 + g + 8];
        } else {
            const double2 lo = *reinterpret_cast<const double2 *>(P + (x0 + g) * QX + kk);
            const double2 hi = *reinterpret_cast<const double2 *>(P + (x0 + g + 8) * QX + kk);
            a[0] = lo.x;
            a[2] = lo.y;
            a[1] = hi.x;
            a[3] = hi.y;
        }
    }
    __device__ __forceinline__ static void ldB(double (&b)[2], const double *P, bool km, int ks, int x0, int g, int t)
    {
        const int kk = ks * 8 + 2 * t;
        if (km) {
            b[0] = P[kk * Pitch<8>::PK + x0 + g];
            b[1] = P[(kk + 1) * Pitch<8>::PK + x0 + g];
        } else {
            const double2 v = *reinterpret_cast<const double2 *>(P + (x0 + g) * QX + kk);
            b[0] = v.x;
            b[1] = v.y;
        }
    }
    __device__ __forceinline__ static void mma(double (&d)[4], const double (&a)[4], const double (&b)[2])
    {
        dmma_16x8x8(d, a, b);
    }
};

// ------------------------------------------------------------------------------------------------
// staging
// ------------------------------------------------------------------------------------------------
template <int K, int VEC>
__device__ __forceinline__ void load_chunk(double *stage, const ItemCtx &cx, int ch, int tid)
{
    const int ph = ch < cx.nV ? 0 : 1;
    const int kk0 = (ph ? ch - cx.nV : ch) * DK;
    const int klim = ph ? cx.nocc : cx.nvir;
    constexpr int CPP = T * DK / VEC;  // copies per panel
    constexpr int ITER = NPANEL * CPP / NTHREAD;
    static_assert(NPANEL * CPP % NTHREAD == 0, "copies must split evenly over the CTA");
#pragma unroll
    for (int u = 0; u < ITER; ++u) {
        const int id = tid + u * NTHREAD;
        const int p = id / CPP;
        const int q = id % CPP;
        if (cx.diag && (p & 1)) continue;  // diagonal pair: the C panels equal the B panels
        const PanelInfo &pi = cx.tbl[ph][p];
        double *dst = stage + p * PANEL;
        const double *src;
        bool ok;
        if (pi.kmajor) {
            const int kk = q / (T / VEC), r = (q % (T / VEC)) * VEC;
            ok = (r < pi.rem) && (kk0 + kk < klim);
            src = pi.base + r + (size_t)(kk0 + kk) * pi.ld;
            dst += kk * Pitch<K>::PK + r;
        } else {
            const int cc = q / (DK / VEC), d = (q % (DK / VEC)) * VEC;
            ok = (cc < pi.rem) && (kk0 + d < klim);
            src = pi.base + (kk0 + d) + (size_t)cc * pi.ld;
            dst += cc * QX + d;
        }
        if (!ok) src = cx.eorb;  // mapped address; zero fill reads nothing
        if (VEC == 2)
            cp_async_16(dst, src, ok);
        else
            cp_async_8(dst, src, ok);
    }
}

// Prepares the context of the next work item (warp 0).  Takes a ticket; state -1 marks the end.
__device__ __forceinline__ void prepare_item(const trpdrv_dev_system *__restrict__ sys, int nsys, long long total,
                                             unsigned long long *counter, ItemCtx &cx, int *status, int lane)
{
    long long item = 0;
    if (lane == 0) item = (long long)atomicAdd(counter, 1ULL);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total) {
        if (lane == 0) cx.state = -1;
        return;
    }
    int s = 0;
    while (s + 1 < nsys && item >= sys[s + 1].item_begin) ++s;
    const trpdrv_dev_system &S = sys[s];
    const long long local = item - S.item_begin;
    const long long qpos = local / S.npairs;  // processing position over the system's records
    const int p = (int)(local - qpos * S.npairs);
    // a index (records are [a][triple], fewer than 2^31: the host checks); no division for a single a
    const long long ai = (S.nt > 0 && qpos >= S.nt) ? (long long)((unsigned)qpos / (unsigned)S.nt) : 0;
    const long long tpos = qpos - ai * S.nt;
    const long long tt = (S.order && local >= 0 && qpos < S.ntriples) ? (long long)S.order[tpos] : tpos;
    const long long own = (ai * S.nt + tt) * S.npairs + p;  // energies go to the record's own items
    int B = 0, rem = p;
    while (B < S.nb && rem >= S.nb - B) {
        rem -= S.nb - B;
        ++B;
    }
    const int C = B + rem;
    const int O = S.nocc, V = S.nvir;
    const bool in_range = local >= 0 && qpos < S.ntriples && tt >= 0 && tt < S.nt && ai < S.n_a;
    const int packed = in_range ? S.triples[tt] : 0;
    const int i = packed & 1023, j = (packed >> 10) & 1023, k = (packed >> 20) & 1023;
    const bool ok = in_range && B < S.nb && C < S.nb && i < O && j < O && k < O && k <= i;
    if (!ok) {
        if (lane == 0) {
            atomicExch(status, 1);
            cx.state = 0;
            cx.out = in_range ? S.partial + (size_t)own * NWARP * 4 : nullptr;
            cx.nch = 0;
        }
        return;
    }
    const size_t lnvv = (size_t)V * V, lnov = (size_t)O * V;
    const size_t jo = (size_t)j * O, ao = (size_t)ai * O;  // ao: the a block of J, K and the vectors
    const int B0 = B * T, C0 = C * T;
    {
        const int ph = lane >> 4, pnl = lane & 15, fam = pnl >> 3, q = pnl & 7;
        const double *Aj, *Ak, *B1, *B3;
        if (fam == 0) {
            Aj = ph ? S.ntov + (size_t)i * lnov : S.jvv + (ao + i) * lnvv;
            Ak = ph ? S.nxov + (size_t)i * lnov : S.kvv + (ao + i) * lnvv;
            B1 = ph ? S.kov + (jo + k) * lnov : S.t2 + (jo + k) * lnvv;
            B3 = ph ? S.jov + (jo + k) * lnov : S.t2 + (jo + k) * lnvv;
        } else {
            Aj = ph ? S.ntov + (size_t)k * lnov : S.jvv + (ao + k) * lnvv;
            Ak = ph ? S.nxov + (size_t)k * lnov : S.kvv + (ao + k) * lnvv;
            B1 = ph ? S.kov + (jo + i) * lnov : S.t2 + (jo + i) * lnvv;
            B3 = ph ? S.jov + (jo + i) * lnov : S.t2 + (jo + i) * lnvv;
        }
        PanelInfo pi;
        pi.pad = 0;
        if (q < 4) {  // A rows: q = 0 A_J rows B, 1 A_J rows C, 2 A_K rows B, 3 A_K rows C
            const int off = (q & 1) ? C0 : B0;
            pi.base = ((q >> 1) ? Ak : Aj) + off;
            pi.ld = V;
            pi.rem = V - off;
            pi.kmajor = 1;
        } else {      // B columns: q = 4 B_1 cols C, 5 B_1 cols B, 6 B_3 cols C, 7 B_3 cols B
            const int off = (q & 1) ? B0 : C0;
            pi.rem = V - off;
            if (q < 6) {  // [T^T ; K]: T(c,d) has c contiguous; K(m,c) has m contiguous
                if (ph == 0) {
                    pi.base = B1 + off;
                    pi.ld = V;
                    pi.kmajor = 1;
                } else {
                    pi.base = B1 + (size_t)off * O;
                    pi.ld = O;
                    pi.kmajor = 0;
                }
            } else {      // [T ; J]: the contraction index is contiguous in both parts
                pi.base = B3 + (size_t)off * (ph ? O : V);
                pi.ld = ph ? O : V;
                pi.kmajor = 0;
            }
        }
        cx.tbl[ph][pnl] = pi;
    }
    if (lane == 0) {
        cx.eorb = S.eorb;
        cx.dintc1 = S.dintc + (ao + i) * V;
        cx.dintx1 = S.dintx + (ao + i) * V;
        cx.t1v1 = S.t1v + (ao + i) * V;
        cx.dintc2 = S.dintc + (ao + k) * V;
        cx.dintx2 = S.dintx + (ao + k) * V;
        cx.t1v2 = S.t1v + (ao + k) * V;
        cx.out = S.partial + (size_t)own * NWARP * 4;
        // omp/ccsd_trpdrv_omp_cbody.c:126 (a is 1-based, i/j/k here 0-based)
        cx.eaijk = S.eorb[S.a - 1 + ai] - (S.eorb[S.ncor + i] + S.eorb[S.ncor + j] + S.eorb[S.ncor + k]);
        cx.ncor = S.ncor;
        cx.nocc = O;
        cx.nvir = V;
        cx.b0 = B0;
        cx.c0 = C0;
        cx.diag = (B == C);
        cx.nV = (V + DK - 1) / DK;
        cx.nO = (O + DK - 1) / DK;
        cx.nch = cx.nV + cx.nO;
        cx.state = 1;
    }
}

// ------------------------------------------------------------------------------------------------
// energies of one warp's sub-block, in registers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void warp_epilogue(const ItemCtx &cx, const double (&f)[8][4], const double (&gT)[8][4],
                                              int rb0, int cb0, int g, int t, int lane, double *out)
{
    TengySums su = {0.0, 0.0, 0.0, 0.0};
    const int V = cx.nvir, voff = cx.ncor + cx.nocc;
    const double eaijk = cx.eaijk;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int b = rb0 + g + ((e & 2) ? 8 : 0);
        const int c = cb0 + 2 * t + (e & 1);
        if (b < V && c < V) {
            double fbc[8], fcb[8];
#pragma unroll
            for (int x = 0; x < 8; ++x) {
                fbc[x] = f[x][e];
                fcb[x] = gT[x][e];
            }
            const double eb = __ldg(cx.eorb + voff + b), ec = __ldg(cx.eorb + voff + c);
            // term at (b,c): omp/ccsd_tengy_c99.c:65 denominator, :91-111 forms
            tengy_term(fbc, fcb, -1.0 / (eb + ec + eaijk), __ldg(cx.t1v1 + b), __ldg(cx.t1v2 + b),
                       __ldg(cx.dintx1 + c), __ldg(cx.dintx2 + c), __ldg(cx.dintc1 + c), __ldg(cx.dintc2 + c), su);
            if (!cx.diag)  // term at (c,b) of the mirrored tile
                tengy_term(fcb, fbc, -1.0 / (ec + eb + eaijk), __ldg(cx.t1v1 + c), __ldg(cx.t1v2 + c),
                           __ldg(cx.dintx1 + b), __ldg(cx.dintx2 + b), __ldg(cx.dintc1 + b), __ldg(cx.dintc2 + b),
                           su);
        }
    }
    su.e4i = warp_sum(su.e4i);
    su.e5i = warp_sum(su.e5i);
    su.e4k = warp_sum(su.e4k);
    su.e5k = warp_sum(su.e5k);
    if (lane == 0 && out) {
        out[0] = su.e4i;
        out[1] = su.e5i;
        out[2] = su.e4k;
        out[3] = su.e5k;
    }
}

// ------------------------------------------------------------------------------------------------
template <int K, int VEC>
__global__ void __launch_bounds__(NTHREAD, 1)
fused_kernel(const trpdrv_dev_system *__restrict__ sys, int nsys, long long total, unsigned long long *counter,
             int *status)
{
    using M = Mma<K>;
    extern __shared__ __align__(16) double smem[];
    __shared__ ItemCtx ring[RING];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    // sub-block of this warp: rows (b) rs*16.., columns (c) cs*8..; the two warps sharing a
    // scheduler (warp, warp+4) differ in both, so padding at a ragged edge idles no scheduler entirely
    const int rs = warp >> 2, cs = (warp & 3) ^ (rs << 1);
    const int rx0 = rs * 16, cx0 = cs * 8;

    // uniform pipeline state (identical in every thread)
    int n_prep = 0;              // items whose context has been prepared
    int n_load = 0, c_load = 0;  // item / chunk the next load reads
    int n_comp = 0, c_comp = 0;  // item / chunk the next compute consumes
    long long g_load = 0, g_comp = 0;  // chunks loaded / consumed (stage = count % STAGES)

    double f[8][4], gT[8][4];
#pragma unroll
    for (int x = 0; x < 8; ++x)
#pragma unroll
        for (int e = 0; e < 4; ++e) f[x][e] = gT[x][e] = 0.0;

    // loads the next chunk (if any) and commits one cp.async group either way
    auto load_next = [&]() {
        while (true) {
            if (n_load >= n_prep) break;  // not prepared yet
            const ItemCtx &cl = ring[n_load % RING];
            if (cl.state < 0) break;      // end of work
            if (cl.state == 0 || c_load >= cl.nch) {  // nothing (more) to load from this item
                if (n_load + 1 >= n_prep) break;
                ++n_load;
                c_load = 0;
                continue;
            }
            load_chunk<K, VEC>(smem + (g_load % STAGES) * STAGE, cl, c_load, tid);
            ++g_load;
            ++c_load;
            break;
        }
        cp_async_commit();
    };
    // warp 0 prepares the context after the newest one when the load side will need it next
    auto maybe_prepare = [&]() {
        if (n_prep > 0 && ring[(n_prep - 1) % RING].state < 0) return;  // end reached
        if (n_prep <= n_load + 1 && n_prep < n_comp + RING - 1) {
            if (warp == 0) prepare_item(sys, nsys, total, counter, ring[n_prep % RING], status, lane);
            ++n_prep;
        }
    };

    // prologue: contexts and the first STAGES-1 chunks
    for (int s = 0; s < STAGES - 1; ++s) {
        maybe_prepare();
        __syncthreads();
        load_next();
    }

    for (;;) {
        maybe_prepare();
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        if (n_comp >= n_prep) break;
        const ItemCtx &cx = ring[n_comp % RING];
        if (cx.state < 0) break;
        if (cx.state == 0) {  // malformed queue entry: zero energies, no chunks
            if (lane == 0 && cx.out) {
                double *o = cx.out + warp * 4;
                o[0] = o[1] = o[2] = o[3] = 0.0;
            }
            ++n_comp;
            c_comp = 0;
            load_next();
            continue;
        }
        load_next();

        const double *st = smem + (g_comp % STAGES) * STAGE;
        const bool ph1 = c_comp >= cx.nV;
        const bool active = (cx.b0 + rx0 < cx.nvir) && (cx.c0 + cx0 < cx.nvir);
        if (active) {
            const int o1 = cx.diag ? 0 : 1;  // diagonal pair: the C panels are the B panels
#pragma unroll
            for (int ks = 0; ks < DK / K; ++ks) {
#pragma unroll
                for (int fam = 0; fam < 2; ++fam) {
                    const double *P = st + fam * 8 * PANEL;
                    double aJ[M::NA], aK[M::NA], a1[M::NA], a3[M::NA];
                    double bJ[M::NB], bK[M::NB], b1[M::NB], b3[M::NB];
                    // A_J/A_K rows B (MMA A side), A_J/A_K rows C (swapped MMA, B side): K-major
                    M::ldA(aJ, P + 0 * PANEL, true, ks, rx0, g, t);
                    M::ldA(aK, P + 2 * PANEL, true, ks, rx0, g, t);
                    M::ldB(bJ, P + (0 + o1) * PANEL, true, ks, cx0, g, t);
                    M::ldB(bK, P + (2 + o1) * PANEL, true, ks, cx0, g, t);
                    // B_1/B_3 columns C (B side) and columns B (swapped MMA, A side)
                    M::ldB(b1, P + 4 * PANEL, !ph1, ks, cx0, g, t);
                    M::ldB(b3, P + 6 * PANEL, false, ks, cx0, g, t);
                    M::ldA(a1, P + (4 + o1) * PANEL, !ph1, ks, rx0, g, t);
                    M::ldA(a3, P + (6 + o1) * PANEL, false, ks, rx0, g, t);
                    const int x0 = fam * 4;
                    // f1 = A_J B_1, f2 = A_K B_1, f3 = A_J B_3, f4 = A_K B_3
                    M::mma(f[x0 + 0], aJ, b1);
                    M::mma(f[x0 + 1], aK, b1);
                    M::mma(f[x0 + 2], aJ, b3);
                    M::mma(f[x0 + 3], aK, b3);
                    // transposes: f_x(c,b) = sum_d B_x(d,b) A_x(c,d)
                    M::mma(gT[x0 + 0], a1, bJ);
                    M::mma(gT[x0 + 1], a1, bK);
                    M::mma(gT[x0 + 2], a3, bJ);
                    M::mma(gT[x0 + 3], a3, bK);
                }
            }
        }
        ++g_comp;
        ++c_comp;
        if (c_comp >= cx.nch) {
            warp_epilogue(cx, f, gT, cx.b0 + rx0, cx.c0 + cx0, g, t, lane, cx.out ? cx.out + warp * 4 : nullptr);
#pragma unroll
            for (int x = 0; x < 8; ++x)
#pragma unroll
                for (int e = 0; e < 4; ++e) f[x][e] = gT[x][e] = 0.0;
            ++n_comp;
            c_comp = 0;
        }
    }
    cp_async_wait<0>();
}

template <int K, int VEC>
int launch(const trpdrv_dev_system *d_sys, int nsys, int64_t total, unsigned long long *counter, int *status,
           int grid, cudaStream_t st)
{
    fused_kernel<K, VEC><<<grid, NTHREAD, SMEM_BYTES, st>>>(d_sys, nsys, total, counter, status);
    return (int)cudaGetLastError();
}

template <int K, int VEC>
int set_smem()
{
    return (int)cudaFuncSetAttribute(fused_kernel<K, VEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)SMEM_BYTES);
}

}  // namespace fused
}  // namespace trpdrv

using namespace trpdrv;

extern "C" size_t trpdrv_fused_smem_bytes(void) { return fused::SMEM_BYTES; }
extern "C" int trpdrv_fused_threads(void) { return fused::NTHREAD; }

extern "C" int trpdrv_fused_max_ctas_per_sm(int *n)
{
    return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, fused::fused_kernel<8, 2>, fused::NTHREAD,
                                                              fused::SMEM_BYTES);
}

extern "C" int trpdrv_launch_fused(const trpdrv_dev_system *d_sys, int nsys, int64_t total_items,
                                   unsigned long long *counter, int *status, int grid, int vec2, int mma_k,
                                   void *stream)
{
    if (grid <= 0 || total_items <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    if (mma_k == 4)
        return vec2 ? fused::launch<4, 2>(d_sys, nsys, total_items, counter, status, grid, st)
                    : fused::launch<4, 1>(d_sys, nsys, total_items, counter, status, grid, st);
    return vec2 ? fused::launch<8, 2>(d_sys, nsys, total_items, counter, status, grid, st)
                : fused::launch<8, 1>(d_sys, nsys, total_items, counter, status, grid, st);
}

extern "C" int trpdrv_fused_init(void)
{
    int e = fused::set_smem<4, 1>();
    if (!e) e = fused::set_smem<4, 2>();
    if (!e) e = fused::set_smem<8, 1>();
    if (!e) e = fused::set_smem<8, 2>();
    return e;
}
