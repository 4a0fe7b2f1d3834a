// Fused persistent triples kernel, TMA + mbarrier pipeline (sm_100a, FP64 DMMA).
//
// Same work decomposition and register-resident energy epilogue as fused.cu (a work item is
// (triple, tile pair {B,C}); each consumer warp owns a 16(b) x 8(c) sub-block and computes all eight
// f of omp/ccsd_trpdrv_omp_cbody.c:70-117 at (b,c) and, through the operand-swapped MMA, at (c,b)),
// but the operand panels are staged by the Tensor Memory Accelerator:
//
//  * one producer thread takes work tickets, writes each item's context to a ring in shared memory
//    and issues, per chunk of DK contraction indices, one or two cp.async.bulk.tensor loads per
//    panel (each CTA loads its own copy) that complete on the stage's "full" mbarrier;
//  * eight consumer warps wait on "full", run the m16n8k8 DMMAs straight from the staged panels and
//    release the stage through its "empty" mbarrier; no CTA-wide barrier in the main loop.
//
// Panel layouts in shared memory (4 KB per panel, 16 panels per stage, DK = 16):
//  * K-major panels (rows contiguous in HBM: Jia/Kia/Jka/Kka, -Tia/-Xia/-Tka/-Xka, T2 as T(c,d)):
//    two 16-row boxes of [DK][16] doubles written with the 128-byte swizzle, which makes the
//    k-permuted fragment reads bank-conflict free;
//  * X-major panels (contraction contiguous: T2 as T(d,c), Jkj/Kkj/Jij/Kij): one [32][DK] box, also
//    128-byte swizzled, read with 128-bit loads.
// Every box row is a full 128-byte line: with 64-byte rows (DK = 8) the TMA request rate, not L2
// bandwidth, bounded the staging at about half of this rate.
// Fragment row/column labels are permuted, lane group g owning row (and column) PERM[g] of its 8,
// PERM = {0,6,1,7,2,4,3,5}: the two rows a quarter-warp reads with one 128-bit load of an X-major
// panel then differ in bit 2 (disjoint bank sets under the 128-byte swizzle) and the rows of one
// 64-bit load of a K-major panel differ in bit 1 where they share bit 0, so no fragment read has a
// bank conflict.  The permutation only relabels which (b, c) a register holds; the epilogue and the
// diagonal exchange use the permuted coordinates.
// The MMA shape is a template parameter: m16n8k8 (two k-steps per 16-index chunk) or m16n8k16,
// whose fragments are exactly the two k8 fragments of the chunk side by side (lane t holds logical
// k = t + 4q at physical index 2t + (q & 1) + 8 (q >> 1)).
// The 3-D tensor maps ([system block][contraction][row]) give every dimension its own bound, so the
// ragged tails in nvir and nocc are zero-filled by the TMA unit.
//
// Every wait is bounded (globaltimer); a wait that runs out sets bit 1 of *status and the CTA stops
// issuing work.  Requires even nvir and nocc and 16-byte aligned tensors (host checks).

#include <cuda.h>
#include <cudaTypedefs.h>

#include "device_common.cuh"
#include "launch.h"

namespace trpdrv {
namespace tma {

constexpr int T = TRPDRV_TILE;  // 32
constexpr int DK = 16;          // contraction indices per stage (two m16n8k8 steps; 128-byte box rows)
constexpr int STAGES = 3;
constexpr int NCW = TRPDRV_FUSED_SLOTS;  // consumer warps (8) = two warpgroups
constexpr int NTHREAD = (NCW + 4) * 32;  // + one producer warpgroup (one thread issues)
// Register split by setmaxnreg: launched at 65536 / 384 = 168 per thread; the producer warpgroup
// drops and the two consumer warpgroups rise, within 384 * 168 = 64512: the m16n8k16 kernel's MMA
// warps take 224 (producer 56: 2*128*224 + 128*56 = 64512), the m16n8k8 kernel's 216 (producer 64),
// the splits under which neither kernel's MMA loop spills.
constexpr int REG_LAUNCH = 168;
template <int KS> struct Regs {
    static constexpr int CONSUMER = KS == 16 ? 224 : 216, PRODUCER = KS == 16 ? 56 : 64;
    static_assert(2 * 128 * CONSUMER + 128 * PRODUCER <= NTHREAD * REG_LAUNCH, "register split exceeds the launch");
};
constexpr int PANEL_BYTES = 4096;
constexpr int NPANEL = 16;
constexpr int STAGE_BYTES = NPANEL * PANEL_BYTES;
constexpr int RING = 16;
constexpr int XBUF = T * (T + 1);  // one padded 32x32 f tile
constexpr int KBOX = PANEL_BYTES / 2;  // one 16-row K-major box
constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_BYTES + 1024;  // + alignment slack
constexpr unsigned long long WAIT_LIMIT_NS = 4000000000ull;       // 4 s: far above any legitimate wait

static_assert(RING >= STAGES + 2, "context ring too small");

enum { M_J = 0, M_K, M_NT, M_NX, M_T2K, M_T2X, M_JOV, M_KOV, NMAP };

struct __align__(64) Maps {
    CUtensorMap m[TRPDRV_TMA_MAX_SYSTEMS][NMAP];
};

struct ItemCtx {
    const double *eorb, *dintc1, *dintx1, *t1v1, *dintc2, *dintx2, *t1v2;
    double *out, *out1;  // energy slots of the item's pair (and of the second pair of a packed item)
    double eaijk;
    int ncor, nocc, nvir, b0, c0, diag, nV, nch, state;  // state: 1 work, 0 malformed, -1 end
    int packed, b1;      // packed edge item: pairs (b0, c0) and (b1, c0); b1 < 0 when the second is absent
    // split item (the one-triple system of a split launch): 1 | half << 1 | pair << 2, else 0; this half
    // runs chunks half, half + 2, ...  One int keeps the context at 128 bytes: at 160 bytes (the split
    // fields as separate members) the batched kernel measured 6 % slower.
    int split_tag;
};

static_assert(sizeof(ItemCtx) == 128, "the item context is kept at 128 bytes (see split_tag)");

// Packed edge items (systems with pack_edge: the last column tile E holds 1..16 valid indices).  The
// pairs (B, E) and (B + 1, E), B even, run as one item: each family of a chunk gets its own stage
// slot, in which the 4 KB panels are
//   0, 1: J (or -T) rows of B and B + 1      2, 3: K (or -X) rows of B and B + 1   (K-major, 2 boxes)
//   4: B_1 columns of E (1 K-major box, or 1 X-major box)   5: B_3 columns of E (X-major)
//   6, 7: J / K (or -T / -X) rows of E (1 K-major box each)
//   8, 9: B_1 columns of B and B + 1 (2 K-major boxes, or 1 X-major)   10, 11: B_3 columns (X-major)
// and warp w computes pair w >> 2, rows 16 ((w & 3) >> 1) and columns 8 (w & 1) of it: the work of one
// full pair over 8 warps instead of two half-idle pairs.
constexpr int PK_A = 0, PK_B1E = 4, PK_B3E = 5, PK_AE = 6, PK_B1B = 8, PK_B3B = 10;

// ------------------------------------------------------------------------------------------------
// PTX helpers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count)
{
    asm volatile("mbarrier.init.shared.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *b, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *b)
{
    asm volatile("mbarrier.arrive.shared.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *b, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity; false (and status bit 1) when it runs out.
// try_wait itself suspends the warp for a while in hardware; the clock is read only every 256
// failed polls so that waiting warps take few issue slots from the MMA warps of their scheduler.
__device__ __forceinline__ bool mbar_wait_for(unsigned long long *b, unsigned parity, int *status,
                                              unsigned long long limit_ns)
{
    if (mbar_try_wait(b, parity)) return true;
    const unsigned long long t0 = globaltimer();
    for (;;) {
#pragma unroll 1
        for (int spin = 0; spin < 256; ++spin)
            if (mbar_try_wait(b, parity)) return true;
        if (globaltimer() - t0 > limit_ns) {
            atomicOr(status, 2);
            return false;
        }
    }
}

__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity, int *status)
{
    return mbar_wait_for(b, parity, status, WAIT_LIMIT_NS);
}

// Self-test of the bounded waits: one thread waits, with the given limit, on an mbarrier that
// nothing completes; the wait must give up, set status bit 1 and return (elapsed_ns: how long it took).
__global__ void bounded_wait_selftest_kernel(unsigned long long limit_ns, int *status,
                                             unsigned long long *elapsed_ns)
{
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const unsigned long long t0 = globaltimer();
    const bool completed = mbar_wait_for(&bar, 0u, status, limit_ns);
    *elapsed_ns = globaltimer() - t0;
    if (completed) atomicOr(status, 4);  // a phase nothing arrived on reported complete
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, unsigned long long *bar, int x, int y,
                                            int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(saddr(dst)), "l"(map), "r"(saddr(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// ------------------------------------------------------------------------------------------------
// fragments (m16n8k8, lane t holds logical k = t and t+4 at physical kk = 2t, 2t+1)
// ------------------------------------------------------------------------------------------------
// Byte offsets of one thread's fragment elements inside a staged panel.  They depend only on the
// thread's sub-block and lane, so they are computed once and every fragment read in the main loop is
// a single shared load at (panel base + constant offset).
// Row/column of its 8 that lane group g (0..7) owns (see the header): conflict-free fragment reads.
__device__ __forceinline__ int perm8(int g) { return (0x53427160 >> (4 * g)) & 7; }

__device__ __forceinline__ int kmajor_off(int kk, int x)
{
    const int h = x >> 4, xi = x & 15;
    return h * KBOX + kk * 128 + (((xi >> 1) ^ (kk & 7)) << 4) + ((xi & 1) << 3);
}

struct FragOffsets {
    int kA0, kA1, kA2, kA3;  // K-major A fragment: (2t, r), (2t, r+8), (2t+1, r), (2t+1, r+8)
    int kB0, kB1;            // K-major B fragment: (2t, c), (2t+1, c)
    int xA0, xA1;            // X-major A fragment: rows r, r+8 at contraction 2t (128-bit)
    int xB;                  // X-major B fragment: column c at contraction 2t (128-bit)
    __device__ __forceinline__ FragOffsets(int rx0, int cx0, int g, int t)
    {
        const int r = rx0 + perm8(g), c = cx0 + perm8(g);
        kA0 = kmajor_off(2 * t, r);
        kA1 = kmajor_off(2 * t, r + 8);
        kA2 = kmajor_off(2 * t + 1, r);
        kA3 = kmajor_off(2 * t + 1, r + 8);
        kB0 = kmajor_off(2 * t, c);
        kB1 = kmajor_off(2 * t + 1, c);
        xA0 = r * 128 + ((t ^ (r & 7)) << 4);
        xA1 = (r + 8) * 128 + ((t ^ ((r + 8) & 7)) << 4);
        xB = c * 128 + ((t ^ (c & 7)) << 4);
    }
    __device__ __forceinline__ static double ld(const char *p, int off) { return *reinterpret_cast<const double *>(p + off); }
    __device__ __forceinline__ static double2 ld2(const char *p, int off) { return *reinterpret_cast<const double2 *>(p + off); }
    __device__ __forceinline__ void ldA_K(double (&a)[4], const char *P) const
    {
        a[0] = ld(P, kA0);
        a[1] = ld(P, kA1);
        a[2] = ld(P, kA2);
        a[3] = ld(P, kA3);
    }
    __device__ __forceinline__ void ldB_K(double (&b)[2], const char *P) const
    {
        b[0] = ld(P, kB0);
        b[1] = ld(P, kB1);
    }
    __device__ __forceinline__ void ldA_X(double (&a)[4], const char *P, int kx) const
    {
        const double2 lo = ld2(P, xA0 ^ kx), hi = ld2(P, xA1 ^ kx);
        a[0] = lo.x;
        a[2] = lo.y;
        a[1] = hi.x;
        a[3] = hi.y;
    }
    __device__ __forceinline__ void ldB_X(double (&b)[2], const char *P, int kx) const
    {
        const double2 v = ld2(P, xB ^ kx);
        b[0] = v.x;
        b[1] = v.y;
    }
};

// m16n8k16 fragments: the k8 fragments of the chunk's two k-steps (K-major panels: the second
// k-step starts 8 rows = 1024 bytes further; X-major panels: 64 bytes further in each row).
__device__ __forceinline__ void ld_a16_K(const FragOffsets &fo, double (&a)[8], const char *P)
{
    fo.ldA_K(*reinterpret_cast<double(*)[4]>(&a[0]), P);
    fo.ldA_K(*reinterpret_cast<double(*)[4]>(&a[4]), P + 1024);
}
__device__ __forceinline__ void ld_b16_K(const FragOffsets &fo, double (&b)[4], const char *P)
{
    fo.ldB_K(*reinterpret_cast<double(*)[2]>(&b[0]), P);
    fo.ldB_K(*reinterpret_cast<double(*)[2]>(&b[2]), P + 1024);
}
__device__ __forceinline__ void ld_a16_X(const FragOffsets &fo, double (&a)[8], const char *P)
{
    fo.ldA_X(*reinterpret_cast<double(*)[4]>(&a[0]), P, 0);
    fo.ldA_X(*reinterpret_cast<double(*)[4]>(&a[4]), P, 64);
}
__device__ __forceinline__ void ld_b16_X(const FragOffsets &fo, double (&b)[4], const char *P)
{
    fo.ldB_X(*reinterpret_cast<double(*)[2]>(&b[0]), P, 0);
    fo.ldB_X(*reinterpret_cast<double(*)[2]>(&b[2]), P, 64);
}

// One family's products of a packed edge item in one stage slot (layout at PK_*): this warp's
// sub-block of pair pp, f_x(b,c) = A_x(b,.) B_x(.,c) and f_x(c,b) through the operand-swapped MMA,
// exactly as the normal items compute them from their o = 0 / o = 1 panels.
template <int KS, int FAM>
__device__ __forceinline__ void packed_family(const FragOffsets &fo, const char *st, int pp, bool ph1, int kval,
                                              double (&f)[8][4], double (&gT)[8][4])
{
    constexpr int x0 = FAM * 4;
    const char *AJ = st + (PK_A + pp) * PANEL_BYTES, *AK = st + (PK_A + 2 + pp) * PANEL_BYTES;
    const char *B1 = st + PK_B1E * PANEL_BYTES, *B3 = st + PK_B3E * PANEL_BYTES;
    const char *AJE = st + PK_AE * PANEL_BYTES, *AKE = st + (PK_AE + 1) * PANEL_BYTES;
    const char *B1B = st + (PK_B1B + pp) * PANEL_BYTES, *B3B = st + (PK_B3B + pp) * PANEL_BYTES;
    if (KS == 16 && kval > 8) {
        double aJ[8], aK[8], b1[4], b3[4];
        ld_a16_K(fo, aJ, AJ);
        ld_a16_K(fo, aK, AK);
        ld_b16_X(fo, b3, B3);
        if (!ph1)
            ld_b16_K(fo, b1, B1);
        else
            ld_b16_X(fo, b1, B1);
        dmma_16x8x16(f[x0 + 0], aJ, b1);
        dmma_16x8x16(f[x0 + 1], aK, b1);
        dmma_16x8x16(f[x0 + 2], aJ, b3);
        dmma_16x8x16(f[x0 + 3], aK, b3);
        double a1[8], a3[8], bJ[4], bK[4];
        ld_b16_K(fo, bJ, AJE);
        ld_b16_K(fo, bK, AKE);
        ld_a16_X(fo, a3, B3B);
        if (!ph1)
            ld_a16_K(fo, a1, B1B);
        else
            ld_a16_X(fo, a1, B1B);
        dmma_16x8x16(gT[x0 + 0], a1, bJ);
        dmma_16x8x16(gT[x0 + 1], a1, bK);
        dmma_16x8x16(gT[x0 + 2], a3, bJ);
        dmma_16x8x16(gT[x0 + 3], a3, bK);
    } else {
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            if (ks == 1 && kval <= 8) break;
            const int kk = ks * 1024, kx = ks * 64;
            double aJ[4], aK[4], b1[2], b3[2];
            fo.ldA_K(aJ, AJ + kk);
            fo.ldA_K(aK, AK + kk);
            fo.ldB_X(b3, B3, kx);
            if (!ph1)
                fo.ldB_K(b1, B1 + kk);
            else
                fo.ldB_X(b1, B1, kx);
            dmma_16x8x8(f[x0 + 0], aJ, b1);
            dmma_16x8x8(f[x0 + 1], aK, b1);
            dmma_16x8x8(f[x0 + 2], aJ, b3);
            dmma_16x8x8(f[x0 + 3], aK, b3);
            double a1[4], a3[4], bJ[2], bK[2];
            fo.ldB_K(bJ, AJE + kk);
            fo.ldB_K(bK, AKE + kk);
            fo.ldA_X(a3, B3B, kx);
            if (!ph1)
                fo.ldA_K(a1, B1B + kk);
            else
                fo.ldA_X(a1, B1B, kx);
            dmma_16x8x8(gT[x0 + 0], a1, bJ);
            dmma_16x8x8(gT[x0 + 1], a1, bK);
            dmma_16x8x8(gT[x0 + 2], a3, bJ);
            dmma_16x8x8(gT[x0 + 3], a3, bK);
        }
    }
}

// Brings the 128-byte lines of the energy vectors the item's epilogue will read into L1 (lanes 0..27:
// 7 vectors x {B, C} block x 2 lines), so the register epilogue does not wait on L2.
__device__ __forceinline__ void prefetch_epilogue(const ItemCtx &cx, int lane)
{
    if (lane >= 28) return;
    const int v = lane >> 2, r = (lane >> 1) & 1, l = lane & 1;
    const double *base;
    switch (v) {
    case 0: base = cx.eorb + cx.ncor + cx.nocc; break;
    case 1: base = cx.t1v1; break;
    case 2: base = cx.t1v2; break;
    case 3: base = cx.dintx1; break;
    case 4: base = cx.dintx2; break;
    case 5: base = cx.dintc1; break;
    default: base = cx.dintc2; break;
    }
    const int idx = (r ? cx.c0 : cx.b0) + 16 * l;
    if (idx < cx.nvir) asm volatile("prefetch.global.L1 [%0];" ::"l"(base + idx));
}

// ------------------------------------------------------------------------------------------------
// energies of one warp's sub-block, in registers (as fused.cu)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void warp_epilogue(const ItemCtx &cx, const double (&f)[8][4], const double (&gT)[8][4],
                                              int rb0, int cb0, int g, int t, int lane, double *out)
{
    TengySums su = {0.0, 0.0, 0.0, 0.0};
    const int V = cx.nvir, voff = cx.ncor + cx.nocc;
    const double eaijk = cx.eaijk;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int b = rb0 + perm8(g) + ((e & 2) ? 8 : 0);
        const int c = cb0 + perm8(2 * t + (e & 1));
        if (b < V && c < V) {
            double fbc[8], fcb[8];
#pragma unroll
            for (int x = 0; x < 8; ++x) {
                fbc[x] = f[x][e];
                fcb[x] = gT[x][e];
            }
            const double eb = __ldg(cx.eorb + voff + b), ec = __ldg(cx.eorb + voff + c);
            // omp/ccsd_tengy_c99.c:65 denominator; e_b + e_c == e_c + e_b, so (b,c) and (c,b) share it
            const double denom = -1.0 / (eb + ec + eaijk);
            // term at (b,c): :91-111 forms
            tengy_term_factored(fbc, fcb, denom, __ldg(cx.t1v1 + b), __ldg(cx.t1v2 + b), __ldg(cx.dintx1 + c),
                                __ldg(cx.dintx2 + c), __ldg(cx.dintc1 + c), __ldg(cx.dintc2 + c), su);
            if (!cx.diag)  // term at (c,b) of the mirrored tile
                tengy_term_factored(fcb, fbc, denom, __ldg(cx.t1v1 + c), __ldg(cx.t1v2 + c), __ldg(cx.dintx1 + b),
                                    __ldg(cx.dintx2 + b), __ldg(cx.dintc1 + b), __ldg(cx.dintc2 + b), su);
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
// producer warp: tickets and item contexts (lane 0), TMA loads (one box per lane)
// ------------------------------------------------------------------------------------------------
// SPLIT: the instantiation that also runs split systems (two work items per pair); without it the
// producer and consumer loops carry no split logic at all.
template <bool SPLIT>
__device__ __forceinline__ void producer(const trpdrv_dev_system *__restrict__ sys, int nsys, long long total,
                                         unsigned long long *counter, int *status, const Maps &maps, char *stages,
                                         unsigned long long *full, unsigned long long *empty, ItemCtx *ring, int lane)
{
    const unsigned FULL = 0xffffffffu;
    // this lane's box within a chunk: group = family*2 + orientation, slot 0..6 (lanes 28..31 idle)
    const int grp = lane / 7, slot = lane - 7 * grp;
    const int fam = grp >> 1, o = grp & 1;
    int stage = 0;
    unsigned phase = 0;  // parity of the current pass over the stages
    long long next = 0;
    if (lane == 0) next = (long long)atomicAdd(counter, 1ULL);
    next = __shfl_sync(FULL, next, 0);
    for (long long n = 0;;) {
        const long long item = next;
        if (item < total) {  // ticket for the following item, early
            if (lane == 0) next = (long long)atomicAdd(counter, 1ULL);
            next = __shfl_sync(FULL, next, 0);
        }
        ItemCtx &cx = ring[n % RING];
        if (item >= total) {
            if (mbar_wait(&empty[stage], phase ^ 1, status) && lane == 0) {
                cx.state = -1;
                mbar_arrive(&full[stage]);
            }
            return;
        }
        int s = 0;
        while (s + 1 < nsys && item >= sys[s + 1].item_begin) ++s;
        const trpdrv_dev_system &S = sys[s];
        // a split system has two work items (halves of the contraction) per pair
        const int hpart = (SPLIT && S.split) ? (int)((item - S.item_begin) & 1) : 0;
        const long long local = (SPLIT && S.split) ? (item - S.item_begin) >> 1 : item - S.item_begin;
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
        // edge pairs (B, E) with B odd are computed by the packed item of B - 1
        const bool pack = S.pack_edge && C == S.nb - 1 && B < C;
        if (pack && (B & 1)) continue;
        const int O = S.nocc, V = S.nvir;
        const bool in_range = local >= 0 && qpos < S.ntriples && tt >= 0 && tt < S.nt && ai < S.n_a;
        const int packed = in_range ? S.triples[tt] : 0;
        const int i = packed & 1023, j = (packed >> 10) & 1023, k = (packed >> 20) & 1023;
        // occupied slots of the i, j and k roles in the tensors (a one-triple system holds two slots)
        const int one = S.one_triple;
        const int zi = one ? 0 : i, zj = one ? 0 : j, zk = one ? 1 : k, zO = one ? 2 : O;
        const bool ok = in_range && B < S.nb && C < S.nb && i < O && j < O && k < O && (one || k <= i) &&
                        (!one || ai == 0) && s < TRPDRV_TMA_MAX_SYSTEMS;
        const int B0 = B * T, C0 = C * T;
        if (!ok) {
            if (!mbar_wait(&empty[stage], phase ^ 1, status)) return;
            if (lane == 0) {
                atomicOr(status, 1);
                cx.state = 0;
                cx.packed = 0;
                cx.out = in_range ? S.partial + (size_t)own * NCW * 4 : nullptr;
                cx.nch = 0;
                mbar_arrive(&full[stage]);
            }
            if (++stage == STAGES) {
                stage = 0;
                phase ^= 1;
            }
            ++n;
            continue;
        }
        const int nV = (V + DK - 1) / DK, nO = (O + DK - 1) / DK;
        const bool diag = (B == C);
        if (lane == 0) {
            cx.eorb = S.eorb;
            const size_t ao = (size_t)ai * zO;  // the a block of the a-dependent vectors
            cx.dintc1 = S.dintc + (ao + zi) * V;
            cx.dintx1 = S.dintx + (ao + zi) * V;
            cx.t1v1 = S.t1v + (ao + zi) * V;
            cx.dintc2 = S.dintc + (ao + zk) * V;
            cx.dintx2 = S.dintx + (ao + zk) * V;
            cx.t1v2 = S.t1v + (ao + zk) * V;
            cx.out = S.partial + (size_t)own * NCW * 4;
            // the second pair (B2, E) of a packed item: its own slots, at its triangular pair index
            // (B2 = B + 1: nb - B - 1 pairs further)
            const bool two = pack && B + 1 < C;
            cx.out1 = cx.out + (two ? (S.nb - B - 1) * NCW * 4 : 0);
            cx.packed = pack;
            cx.b1 = two ? (B + 1) * T : -1;
            // omp/ccsd_trpdrv_omp_cbody.c:126 (a is 1-based, i/j/k here 0-based)
            cx.eaijk = S.eorb[S.a - 1 + ai] - (S.eorb[S.ncor + i] + S.eorb[S.ncor + j] + S.eorb[S.ncor + k]);
            cx.ncor = S.ncor;
            cx.nocc = O;
            cx.nvir = V;
            cx.b0 = B0;
            cx.c0 = C0;
            cx.diag = diag;
            cx.nV = nV;
            cx.split_tag = (SPLIT && S.split) ? 1 | hpart << 1 | (int)own << 2 : 0;
            cx.nch = (SPLIT && S.split) ? (nV + nO - hpart + 1) / 2 : nV + nO;
            cx.state = 1;
        }

        const CUtensorMap *mp = maps.m[s];
        if (pack) {
            // one stage slot per (chunk, family); lanes 0..17 each own at most one box of the layout at
            // PK_*: kind 0 / 1 = J / K-role A rows (K-major), 2 = B_1 columns, 3 = B_3 columns (X-major)
            const int E = C, B2 = B + 1 < C ? B + 1 : -1;
            int kind = 3, tb = -1, half = 0, off = 0;
            if (lane < 8) {
                const int pnl = lane >> 1;
                kind = pnl >> 1;
                tb = (pnl & 1) ? B2 : B;
                half = lane & 1;
                off = (PK_A + pnl) * PANEL_BYTES + half * KBOX;
            } else if (lane < 12) {
                kind = lane == 8 ? 2 : lane == 9 ? 3 : lane - 10;
                tb = E;
                off = (lane == 8 ? PK_B1E : lane == 9 ? PK_B3E : PK_AE + lane - 10) * PANEL_BYTES;
            } else if (lane < 18) {
                const int pp = lane < 16 ? (lane - 12) >> 1 : lane - 16;
                kind = lane < 16 ? 2 : 3;
                tb = pp ? B2 : B;
                half = lane < 16 ? (lane & 1) : 0;
                off = (lane < 16 ? PK_B1B + pp : PK_B3B + pp) * PANEL_BYTES + half * KBOX;
            }
            tb = tb >= 0 ? tb * T : -1;
            const int pch0 = (SPLIT && S.split) ? hpart : 0, pstep = (SPLIT && S.split) ? 2 : 1;
            const int nsl = 2 * ((SPLIT && S.split) ? (nV + nO - hpart + 1) / 2 : nV + nO);
            for (int sl = 0; sl < nsl; ++sl) {
                if (!mbar_wait(&empty[stage], phase ^ 1, status)) return;
                const int fam = sl & 1, ch = pch0 + (sl >> 1) * pstep;
                const bool ph1 = ch >= nV;
                const int kk0 = (ph1 ? ch - nV : ch) * DK;
                const int za = fam ? zk : zi;
                const int zb = fam ? zj * zO + zi : zj * zO + zk;
                const CUtensorMap *m = nullptr;
                int x = kk0, y = tb, z = zb;
                unsigned bytes = 0;
                if (tb >= 0) {
                    if (kind < 2) {  // A rows: J / K (virtual), -T / -X (occupied)
                        m = &mp[ph1 ? (kind ? M_NX : M_NT) : (kind ? M_K : M_J)];
                        x = tb + 16 * half;
                        y = kk0;
                        z = ph1 ? za : za + (int)ai * zO;
                        bytes = KBOX;
                    } else if (kind == 2) {  // B_1 columns: T(c,d) K-major boxes, or one K(m,c) X-major box
                        if (!ph1) {
                            m = &mp[M_T2K];
                            x = tb + 16 * half;
                            y = kk0;
                            bytes = KBOX;
                        } else if (half == 0) {
                            m = &mp[M_KOV];
                            bytes = PANEL_BYTES;
                        }
                    } else {  // B_3 columns: T(d,c) / J(m,c), X-major
                        m = &mp[ph1 ? M_JOV : M_T2X];
                        bytes = PANEL_BYTES;
                    }
                }
                const unsigned total = __reduce_add_sync(FULL, bytes);
                if (lane == 0) mbar_arrive_expect_tx(&full[stage], total);
                __syncwarp();
                if (m) tma_load_3d(stages + (size_t)stage * STAGE_BYTES + off, m, &full[stage], x, y, z);
                if (++stage == STAGES) {
                    stage = 0;
                    phase ^= 1;
                }
            }
            ++n;
            continue;
        }

        // per-lane box: A_J (slots 0,1), A_K (2,3) rows; B_1 (4,5) and B_3 (6) columns
        const int za = fam ? zk : zi;                    // A operands: Jia/Kia (n), Jka/Kka (t)
        const int zaj = za + (int)ai * zO;               // J/K carry the a index, -T/-X do not
        const int zb = fam ? zj * zO + zi : zj * zO + zk;  // B operands: Tkj/Kkj/Jkj (n), Tij/Kij/Jij (t)
        const int ra = o ? C0 : B0;                      // A rows: B for (B,C), C for (C,B)
        const int cb = o ? B0 : C0;                      // B columns: C for (B,C), B for (C,B)
        const int half = slot & 1;                       // second 16-row box of a K-major panel
        const int pnl = fam * 8 + (slot < 2 ? 0 : slot < 4 ? 2 : slot < 6 ? 4 : 6) + o;
        const bool mine = lane < 28 && (!diag || o == 0);
        const unsigned bytes = (diag ? NPANEL / 2 : NPANEL) * PANEL_BYTES;
        for (int ch = (SPLIT && S.split) ? hpart : 0; ch < nV + nO; ch += (SPLIT && S.split) ? 2 : 1) {
            if (!mbar_wait(&empty[stage], phase ^ 1, status)) return;
            if (lane == 0) mbar_arrive_expect_tx(&full[stage], bytes);
            __syncwarp();
            const bool ph1 = ch >= nV;
            const int kk0 = (ph1 ? ch - nV : ch) * DK;
            char *dst = stages + (size_t)stage * STAGE_BYTES + pnl * PANEL_BYTES;
            if (mine) {
                if (slot < 4) {  // A rows, K-major (J/K in the virtual phase, -T/-X in the occupied one)
                    const CUtensorMap *m = &mp[slot < 2 ? (ph1 ? M_NT : M_J) : (ph1 ? M_NX : M_K)];
                    tma_load_3d(dst + half * KBOX, m, &full[stage], ra + 16 * half, kk0, ph1 ? za : zaj);
                } else if (slot < 6) {  // B_1 columns: T(c,d) K-major, or K(m,c) X-major (one box)
                    if (!ph1)
                        tma_load_3d(dst + half * KBOX, &mp[M_T2K], &full[stage], cb + 16 * half, kk0, zb);
                    else if (!half)
                        tma_load_3d(dst, &mp[M_KOV], &full[stage], kk0, cb, zb);
                } else {  // B_3 columns: T(d,c) / J(m,c), X-major
                    tma_load_3d(dst, &mp[ph1 ? M_JOV : M_T2X], &full[stage], kk0, cb, zb);
                }
            }
            if (++stage == STAGES) {
                stage = 0;
                phase ^= 1;
            }
        }
        ++n;
    }
}

// ------------------------------------------------------------------------------------------------
// Split items: both halves write their partial f and f-transposed to scratch (thread-major, so the
// 256 consumer threads write consecutive addresses), make them visible (fence), and one thread counts
// the arrival.  The second half to arrive adds the first's partials and finishes the item (fin = 1);
// the first stops there.  Two rounds of the consumer barrier order the writes before the count and
// broadcast its result; the counter is reset by the second arrival.  Nothing waits for the other CTA.
// Returns false when a barrier wait ran out (status set).
__device__ __forceinline__ bool split_combine(const trpdrv_dev_system *__restrict__ sys, const ItemCtx &cx,
                                              double (&f)[8][4], double (&gT)[8][4], int warp, int lane,
                                              unsigned long long *xbar, unsigned &xphase, int *flag, int *status,
                                              int &fin)
{
    const int tc = warp * 32 + lane, half = (cx.split_tag >> 1) & 1;
    const size_t pair = (size_t)(cx.split_tag >> 2);
    double *const scr = sys[0].split_scratch + pair * 2 * 64 * 256;  // [2 halves][64][256] of this pair
    unsigned *const cnt = sys[0].split_count + pair;                 // arrivals of the two halves
    double *mine = scr + (size_t)(half ? 64 * 256 : 0) + tc;
#pragma unroll
    for (int x = 0; x < 8; ++x)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            mine[(x * 4 + e) * 256] = f[x][e];
            mine[(32 + x * 4 + e) * 256] = gT[x][e];
        }
    __threadfence();
    __syncwarp();
    if (lane == 0) mbar_arrive(xbar);
    if (!mbar_wait(xbar, xphase, status)) return false;
    xphase ^= 1;
    if (tc == 0) *flag = (int)atomicAdd(cnt, 1u);
    __syncwarp();
    if (lane == 0) mbar_arrive(xbar);
    if (!mbar_wait(xbar, xphase, status)) return false;
    xphase ^= 1;
    fin = *flag != 0;
    if (fin) {
        __threadfence();
        const double *other = scr + (size_t)(half ? 0 : 64 * 256) + tc;
#pragma unroll
        for (int x = 0; x < 8; ++x)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                f[x][e] += __ldcg(other + (x * 4 + e) * 256);
                gT[x][e] += __ldcg(other + (32 + x * 4 + e) * 256);
            }
        if (tc == 0) *cnt = 0u;
    }
    return true;
}

// ------------------------------------------------------------------------------------------------
template <int KS, bool SPLIT>
__global__ void __launch_bounds__(NTHREAD, 1)
fused_tma_kernel(const trpdrv_dev_system *__restrict__ sys, int nsys, long long total, unsigned long long *counter,
                 int *status, const __grid_constant__ Maps maps)
{
    extern __shared__ char smem_raw[];
    __shared__ __align__(8) unsigned long long full[STAGES], empty[STAGES];
    __shared__ ItemCtx ring[RING];
    __shared__ double xbuf[2 * XBUF];                       // diagonal-pair transpose exchange
    __shared__ __align__(8) unsigned long long xbar[1];
    __shared__ int split_flag[1];
    char *stages = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NCW);
        }
        mbar_init(xbar, NCW);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp >= NCW) {  // producer warpgroup: its first warp issues everything
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(Regs<KS>::PRODUCER));
        if (warp == NCW) producer<SPLIT>(sys, nsys, total, counter, status, maps, stages, full, empty, ring, lane);
        return;
    }
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(Regs<KS>::CONSUMER));

    const int g = lane >> 2, t = lane & 3;
    // sub-block: rows (b) rs*16.., columns (c) cs*8..; warps w and w+4 share a scheduler and differ in both
    const int rs = warp >> 2, cs = (warp & 3) ^ (rs << 1);
    const int rx0 = rs * 16, cx0 = cs * 8;
    const FragOffsets fo(rx0, cx0, g, t);

    double f[8][4], gT[8][4];
    int stage = 0;
    unsigned phase = 0, xphase = 0;
    for (long long n = 0;; ++n) {
        if (!mbar_wait(&full[stage], phase, status)) return;
        const ItemCtx &cx = ring[n % RING];
        const int state = cx.state;
        if (state < 0) return;
        if (state == 0) {
            if (lane == 0 && cx.out) {
                double *o = cx.out + warp * 4;
                o[0] = o[1] = o[2] = o[3] = 0.0;
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[stage]);
            if (++stage == STAGES) {
                stage = 0;
                phase ^= 1;
            }
            continue;
        }
#pragma unroll
        for (int x = 0; x < 8; ++x)
#pragma unroll
            for (int e = 0; e < 4; ++e) f[x][e] = gT[x][e] = 0.0;
        if (cx.packed) {
            // two edge pairs (b0, c0) and (b1, c0): warp w takes pair w >> 2, sub-block w & 3 of it; each
            // (chunk, family) has its own stage slot
            const int pp = warp >> 2, sub = warp & 3, prs = sub >> 1, pcs = sub & 1;
            const FragOffsets fp(prs * 16, pcs * 8, g, t);
            const int pb0 = pp ? cx.b1 : cx.b0;
            const bool pactive = pb0 >= 0 && cx.c0 + pcs * 8 < cx.nvir;
            const int nsl = 2 * cx.nch, pnV = cx.nV;
            // per-item values in registers: every field read after a wait would be reloaded from the ring
            const int inocc = cx.nocc, invir = cx.nvir;
            const int ich0 = SPLIT ? (cx.split_tag >> 1) & 1 : 0, istep = SPLIT ? (cx.split_tag & 1) + 1 : 1;
            for (int sl = 0; sl < nsl; ++sl) {
                if (sl > 0 && !mbar_wait(&full[stage], phase, status)) return;
                const char *st = stages + (size_t)stage * STAGE_BYTES;
                const int ch = ich0 + (sl >> 1) * istep;
                const bool ph1 = ch >= pnV;
                const int kval = ph1 ? inocc - (ch - pnV) * DK : invir - ch * DK;
                if (pactive) {
                    // m16n8k8 here in both kernels: the packed path's extra fragment registers would
                    // push the k16 kernel's MMA warps past their register budget
                    if (sl & 1)
                        packed_family<8, 1>(fp, st, pp, ph1, kval, f, gT);
                    else
                        packed_family<8, 0>(fp, st, pp, ph1, kval, f, gT);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[stage]);
                if (++stage == STAGES) {
                    stage = 0;
                    phase ^= 1;
                }
            }
            if (SPLIT && (cx.split_tag & 1)) {
                int fin = 0;
                if (!split_combine(sys, cx, f, gT, warp, lane, xbar, xphase, split_flag, status, fin)) return;
                if (!fin) continue;
            }
            if (pb0 >= 0) {  // this pair's slots: the 4 sub-blocks' sums, zeros in the other 4
                double *out = pp ? cx.out1 : cx.out;
                warp_epilogue(cx, f, gT, pb0 + prs * 16, cx.c0 + pcs * 8, g, t, lane, out + sub * 4);
                if (lane == 0) {
                    double *z = out + (sub + 4) * 4;
                    z[0] = z[1] = z[2] = z[3] = 0.0;
                }
            }
            continue;
        }
        const int nch = cx.nch, nV = cx.nV;
        // per-item values in registers: every field read after a wait would be reloaded from the ring
        const int inocc = cx.nocc, invir = cx.nvir;
        const int ich0 = SPLIT ? (cx.split_tag >> 1) & 1 : 0, istep = SPLIT ? (cx.split_tag & 1) + 1 : 1;
        const bool active = (cx.b0 + rx0 < cx.nvir) && (cx.c0 + cx0 < cx.nvir);
        const bool diag = cx.diag != 0;
        const int pf = nch > 3 ? nch - 3 : 0;
        for (int c = 0; c < nch; ++c) {
            const int ch = ich0 + c * istep;
            if (c > 0 && !mbar_wait(&full[stage], phase, status)) return;
            const char *st = stages + (size_t)stage * STAGE_BYTES;
            const bool ph1 = ch >= nV;
            // the second k-step of a chunk is skipped when it lies entirely in the zero padding
            const int kval = ph1 ? inocc - (ch - nV) * DK : invir - ch * DK;
            if (c == pf) prefetch_epilogue(cx, lane);
            if (KS == 16 && active && kval > 8) {
                // one m16n8k16 per product: the fragments of both k-steps of the chunk side by side
#pragma unroll
                for (int fam = 0; fam < 2; ++fam) {
                    const char *P = st + fam * 8 * PANEL_BYTES;   // o = 0 panels
                    const char *Q = P + PANEL_BYTES;             // o = 1 panels
                    const int x0 = fam * 4;
                    double aJ[8], aK[8], b1[4], b3[4];
                    ld_a16_K(fo, aJ, P + 0 * PANEL_BYTES);
                    ld_a16_K(fo, aK, P + 2 * PANEL_BYTES);
                    ld_b16_X(fo, b3, P + 6 * PANEL_BYTES);
                    if (!ph1)
                        ld_b16_K(fo, b1, P + 4 * PANEL_BYTES);
                    else
                        ld_b16_X(fo, b1, P + 4 * PANEL_BYTES);
                    dmma_16x8x16(f[x0 + 0], aJ, b1);
                    dmma_16x8x16(f[x0 + 1], aK, b1);
                    dmma_16x8x16(f[x0 + 2], aJ, b3);
                    dmma_16x8x16(f[x0 + 3], aK, b3);
                    if (!diag) {
                        double a1[8], a3[8], bJ[4], bK[4];
                        ld_b16_K(fo, bJ, Q + 0 * PANEL_BYTES);
                        ld_b16_K(fo, bK, Q + 2 * PANEL_BYTES);
                        ld_a16_X(fo, a3, Q + 6 * PANEL_BYTES);
                        if (!ph1)
                            ld_a16_K(fo, a1, Q + 4 * PANEL_BYTES);
                        else
                            ld_a16_X(fo, a1, Q + 4 * PANEL_BYTES);
                        dmma_16x8x16(gT[x0 + 0], a1, bJ);
                        dmma_16x8x16(gT[x0 + 1], a1, bK);
                        dmma_16x8x16(gT[x0 + 2], a3, bJ);
                        dmma_16x8x16(gT[x0 + 3], a3, bK);
                    }
                }
            } else if (active) {
#pragma unroll
                for (int ks = 0; ks < 2; ++ks)
#pragma unroll
                for (int fam = 0; fam < 2; ++fam) {
                    if (ks == 1 && kval <= 8) break;
                    const char *P = st + fam * 8 * PANEL_BYTES + ks * 1024;    // o = 0 panels (K-major k-step)
                    const char *Q = P + PANEL_BYTES;               // o = 1 panels (C side)
                    const char *PX = st + fam * 8 * PANEL_BYTES;   // X-major bases
                    const char *QX = PX + PANEL_BYTES;
                    const int kx = ks * 64;
                    const int x0 = fam * 4;
                    double aJ[4], aK[4], b1[2], b3[2];
                    fo.ldA_K(aJ, P + 0 * PANEL_BYTES);
                    fo.ldA_K(aK, P + 2 * PANEL_BYTES);
                    fo.ldB_X(b3, PX + 6 * PANEL_BYTES, kx);
                    if (!ph1)
                        fo.ldB_K(b1, P + 4 * PANEL_BYTES);
                    else
                        fo.ldB_X(b1, PX + 4 * PANEL_BYTES, kx);
                    // f1 = A_J B_1, f2 = A_K B_1, f3 = A_J B_3, f4 = A_K B_3
                    dmma_16x8x8(f[x0 + 0], aJ, b1);
                    dmma_16x8x8(f[x0 + 1], aK, b1);
                    dmma_16x8x8(f[x0 + 2], aJ, b3);
                    dmma_16x8x8(f[x0 + 3], aK, b3);
                    if (!diag) {  // a diagonal pair gets f(c,b) from the other warps instead (below)
                        double a1[4], a3[4], bJ[2], bK[2];
                        fo.ldB_K(bJ, Q + 0 * PANEL_BYTES);
                        fo.ldB_K(bK, Q + 2 * PANEL_BYTES);
                        fo.ldA_X(a3, QX + 6 * PANEL_BYTES, kx);
                        if (!ph1)
                            fo.ldA_K(a1, Q + 4 * PANEL_BYTES);
                        else
                            fo.ldA_X(a1, QX + 4 * PANEL_BYTES, kx);
                        // transposes: f_x(c,b) = sum_d B_x(d,b) A_x(c,d)
                        dmma_16x8x8(gT[x0 + 0], a1, bJ);
                        dmma_16x8x8(gT[x0 + 1], a1, bK);
                        dmma_16x8x8(gT[x0 + 2], a3, bJ);
                        dmma_16x8x8(gT[x0 + 3], a3, bK);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[stage]);
            if (++stage == STAGES) {
                stage = 0;
                phase ^= 1;
            }
        }
        if (SPLIT && (cx.split_tag & 1)) {  // the second half to arrive adds the first's partial sums and finishes
            int fin = 0;
            if (!split_combine(sys, cx, f, gT, warp, lane, xbar, xphase, split_flag, status, fin)) return;
            if (!fin) continue;
        }
        if (diag) {
            // f(c,b) of a diagonal pair is f at the mirrored position of the same 32x32 block, held
            // by another warp: exchange one f at a time through two alternating shared buffers,
            // separated by a consumer-only mbarrier (bounded wait; no CTA-wide barrier).
#pragma unroll
            for (int x = 0; x < 8; ++x) {
                double *xb = xbuf + (x & 1) * XBUF;
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    xb[(rx0 + perm8(g) + ((e & 2) ? 8 : 0)) * (T + 1) + cx0 + perm8(2 * t + (e & 1))] = f[x][e];
                __syncwarp();
                if (lane == 0) mbar_arrive(xbar);
                if (!mbar_wait(xbar, xphase, status)) return;
                xphase ^= 1;
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    gT[x][e] = xb[(cx0 + perm8(2 * t + (e & 1))) * (T + 1) + rx0 + perm8(g) + ((e & 2) ? 8 : 0)];
            }
        }
        warp_epilogue(cx, f, gT, cx.b0 + rx0, cx.c0 + cx0, g, t, lane, cx.out + warp * 4);
    }
}

// ------------------------------------------------------------------------------------------------
// host side: tensor maps
// ------------------------------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 3-D map over doubles: dims {d0 (contiguous), d1, d2}, box {b0, b1, 1}
// zstride: distance in doubles between consecutive blocks of the third dimension (0 = d0 * d1, packed)
static int make_map(CUtensorMap *m, const double *base, unsigned long long d0, unsigned long long d1,
                    unsigned long long d2, unsigned b0, unsigned b1, bool swizzle, unsigned long long zstride = 0)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) return 1;
    const cuuint64_t dims[3] = {d0, d1, d2};
    const cuuint64_t strides[2] = {d0 * 8ull, (zstride ? zstride : d0 * d1) * 8ull};
    const cuuint32_t box[3] = {b0, b1, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE,
                          swizzle ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 2;
}

}  // namespace tma
}  // namespace trpdrv

using namespace trpdrv;

extern "C" size_t trpdrv_tma_maps_bytes(void) { return sizeof(tma::Maps); }

// Registers per thread the kernel is launched with (read back at init).  The setmaxnreg split is
// only valid when this equals REG_LAUNCH: with fewer, the consumers' increase could never be met.
static int g_launch_regs = -1;

extern "C" int trpdrv_tma_supported(const trpdrv_dev_system *h_sys, int nsys)
{
    if (g_launch_regs != tma::REG_LAUNCH) return 0;
    if (nsys > TRPDRV_TMA_MAX_SYSTEMS || !tma::encode_fn()) return 0;
    for (int s = 0; s < nsys; ++s) {
        const trpdrv_dev_system &S = h_sys[s];
        if ((S.nvir & 1) || (S.nocc & 1)) return 0;  // row strides must be multiples of 16 bytes
        const void *p[] = {S.t2, S.jvv, S.kvv, S.ntov, S.nxov, S.jov, S.kov};
        for (const void *q : p)
            if (((uintptr_t)q) & 15u) return 0;
    }
    return 1;
}

// Packing needs at least two edge pairs and an edge tile of at most 16 valid columns (two 8-wide
// column blocks per pair).  TRPDRV_TMA_PACK_EDGE=0 keeps the edge pairs as ordinary items.
extern "C" int trpdrv_tma_pack_edge(int nvir)
{
    const char *v = getenv("TRPDRV_TMA_PACK_EDGE");
    if (v && v[0] == '0') return 0;
    const int nb = (nvir + tma::T - 1) / tma::T, w = nvir - (nb - 1) * tma::T;
    return nb >= 3 && w >= 1 && w <= 16;
}

extern "C" int trpdrv_tma_prepare(const trpdrv_dev_system *h_sys, int nsys, void *maps_out)
{
    tma::Maps *M = static_cast<tma::Maps *>(maps_out);
    memset(M, 0, sizeof(*M));
    for (int s = 0; s < nsys && s < TRPDRV_TMA_MAX_SYSTEMS; ++s) {
        const trpdrv_dev_system &S = h_sys[s];
        const unsigned long long V = S.nvir, O = S.nocc;
        // occupied slots along the block dimension: nocc (x nocc for the j-blocked tensors), or the
        // two slots (one j block) of a one-triple system
        const unsigned long long X = S.one_triple ? 2 : O, O2 = S.one_triple ? 2 : O * O;
        CUtensorMap *m = M->m[s];
        int e = 0;
        const unsigned long long OA = X * (unsigned long long)(S.n_a > 0 ? S.n_a : 1);
        // a one-triple system may place its two slots of every tensor slot_stride doubles apart
        const unsigned long long zs = S.one_triple ? (unsigned long long)S.slot_stride : 0ull;
        e |= tma::make_map(&m[tma::M_J], S.jvv, V, V, OA, 16, tma::DK, true, zs);    // [a][i][d][b]
        e |= tma::make_map(&m[tma::M_K], S.kvv, V, V, OA, 16, tma::DK, true, zs);
        e |= tma::make_map(&m[tma::M_NT], S.ntov, V, O, X, 16, tma::DK, true, zs);  // [i][m][b]
        e |= tma::make_map(&m[tma::M_NX], S.nxov, V, O, X, 16, tma::DK, true, zs);
        e |= tma::make_map(&m[tma::M_T2K], S.t2, V, V, O2, 16, tma::DK, true, zs);  // [jx][d][c]: T(c,d)
        e |= tma::make_map(&m[tma::M_T2X], S.t2, V, V, O2, tma::DK, 32, true, zs); // [jx][c][d]: T(d,c)
        e |= tma::make_map(&m[tma::M_JOV], S.jov, O, V, O2, tma::DK, 32, true, zs);  // [jx][c][m]
        e |= tma::make_map(&m[tma::M_KOV], S.kov, O, V, O2, tma::DK, 32, true, zs);
        if (e) return e;
    }
    return 0;
}

extern "C" int trpdrv_launch_fused_tma(const trpdrv_dev_system *d_sys, int nsys, int64_t total_items,
                                       unsigned long long *counter, int *status, int grid, const void *maps,
                                       int mma_k, int split, void *stream)
{
    if (grid <= 0 || total_items <= 0) return 0;
    if (g_launch_regs != tma::REG_LAUNCH) return (int)cudaErrorInvalidConfiguration;
    const tma::Maps &m = *static_cast<const tma::Maps *>(maps);
    cudaStream_t st = (cudaStream_t)stream;
    if (split && mma_k == 8)
        tma::fused_tma_kernel<8, true><<<grid, tma::NTHREAD, tma::SMEM_BYTES, st>>>(d_sys, nsys, total_items,
                                                                                   counter, status, m);
    else if (split)
        return (int)cudaErrorInvalidValue;
    else if (mma_k == 16)
        tma::fused_tma_kernel<16, false><<<grid, tma::NTHREAD, tma::SMEM_BYTES, st>>>(d_sys, nsys, total_items,
                                                                                     counter, status, m);
    else if (mma_k == 8)
        tma::fused_tma_kernel<8, false><<<grid, tma::NTHREAD, tma::SMEM_BYTES, st>>>(d_sys, nsys, total_items,
                                                                                    counter, status, m);
    else
        return (int)cudaErrorInvalidValue;
    return (int)cudaGetLastError();
}

extern "C" int trpdrv_launch_wait_selftest(unsigned long long limit_ns, int *status, unsigned long long *elapsed_ns,
                                           void *stream)
{
    tma::bounded_wait_selftest_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(limit_ns, status, elapsed_ns);
    return (int)cudaGetLastError();
}

// Every instantiation must be launched with REG_LAUNCH registers per thread (the setmaxnreg split
// assumes it); g_launch_regs holds the common value, or 0 when they differ.
extern "C" int trpdrv_fused_tma_init(void)
{
    cudaFuncAttributes a[3];
    cudaError_t e = cudaFuncGetAttributes(&a[0], tma::fused_tma_kernel<8, false>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a[1], tma::fused_tma_kernel<16, false>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a[2], tma::fused_tma_kernel<8, true>);
    if (e != cudaSuccess) return (int)e;
    g_launch_regs = a[0].numRegs == a[1].numRegs && a[0].numRegs == a[2].numRegs ? a[0].numRegs : 0;
    const cudaFuncAttribute dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
    e = cudaFuncSetAttribute(tma::fused_tma_kernel<8, false>, dyn, (int)tma::SMEM_BYTES);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(tma::fused_tma_kernel<16, false>, dyn, (int)tma::SMEM_BYTES);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(tma::fused_tma_kernel<8, true>, dyn, (int)tma::SMEM_BYTES);
    return (int)e;
}
