// Emulated-FP64 form of the triples body (sm_100a): Ozaki splitting of every contraction into int8
// digit slices on the 5th-generation tensor cores, exact int32 accumulation in tensor memory, FP64
// recombination; energy denominators and sums stay in native FP64.
//
// Each of the eight f of a triple is one contraction over d = [virtual | occupied]
// (omp/ccsd_trpdrv_omp_cbody.c:70-117 with the occupied A operand negated, as in the fused kernels).
// The emulation:
//  * every row of an A operand and every column of a B operand is scaled by a power of two 2^e chosen
//    so that its largest element has magnitude in [1/4, 1/2), then written as S signed base-128
//    digits x = 2^e * sum_{p=1..S} d_p 2^(-7p) with |d_p| <= 64 (each digit rounded to nearest, so the
//    remainder after S digits is at most 2^(e-7S-1));
//  * products of digit slices with p + q <= S + 1 are accumulated on the tensor cores
//    (tcgen05.mma kind::i8, int32 accumulators in TMEM).  Pairs with equal p + q carry the same
//    weight and share one accumulator; |sum| <= S * dp * 64 * 64 < 2^31, so the integer sums are exact;
//  * the S level sums are recombined in FP64: f = 2^(eA + eB) * sum_L 2^(-7L) C_L.
// f of a batch of triples go to a device buffer (L2-sized) and the batched tengy kernel reduces
// them in FP64 exactly like the plain path (omp/ccsd_tengy_c99.c:5-119).
//
// Operand slices (int8, contraction index d contiguous, zero-padded to dp, a multiple of 32):
//   SA[x][p][r][d]:      r < V: [J(x) | -TOV(x)] row r;       r >= V: [K(x) | -XOV(x)] row r - V
//   SB[j*O+y][p][c][d]:  c < V: [T2[j][y]^T ; KOV[j][y]] col c; c >= V: [T2[j][y] ; JOV[j][y]] col c - V
// The n-group of triple (i, j, k) is SA[i] x SB[j,k] and its t-group SA[k] x SB[j,i]; the 2V x 2V
// product [A1; A2] [B1 | B3] holds the four f of the group in its quadrants:
//   f1n = A1 B1, f2n = A2 B1, f3n = A1 B3, f4n = A2 B3 (and f1t..f4t likewise).
//
// Contraction kernel: persistent, one CTA per SM walking 128 x 64 output tiles of the batch's
// (triple, group) products.  Warp 0 issues TMA loads (64-byte swizzle) of all S digit slices of A and
// B for 64 contraction indices per stage and runs ahead across tiles; warp 1 allocates tensor memory
// and one of its threads issues every MMA (M=128, N=64, K=32) into S level accumulators (S*64
// columns); warps 2-9 wait for a tile's last MMA, drain the accumulators with tcgen05.ld, release
// them to the next tile and then scale and store in FP64 while its MMAs run.  Every wait is bounded
// (globaltimer) and reports through *status; tensor memory is released on every path.

#include <cuda.h>
#include <cudaTypedefs.h>

#include "device_common.cuh"
#include "launch.h"
#include "tengy_tile.cuh"

namespace trpdrv {
namespace oz {

constexpr int BM = 128;         // output rows per tile (TMEM lanes)
constexpr int BN = 64;          // output columns per tile (TMEM columns per level)
constexpr int KC = 64;          // contraction bytes (= int8 indices) per stage
constexpr int KSTEP = 32;       // contraction indices per MMA
constexpr int NREC = 8;         // recombination warps: two per TMEM lane quadrant, 32 columns each
constexpr int NENG = 4;         // energy warps (energies fused into the launch)
// Warpgroup 0: warp 0 TMA, warp 1 MMA + TMEM (warps 2, 3 idle); warpgroups 1, 2 (warps 4 .. 11)
// recombination; warpgroup 3 (warps 12 .. 15) energies.
constexpr int REC0 = 4, ENG0 = REC0 + NREC;
constexpr int NTHREAD = 32 * (ENG0 + NENG);
// Register split by setmaxnreg: launched at 65536 / 512 = 128 per thread, the recombination
// warpgroups rise to 168 (their drain spills below that), the others drop.
constexpr int REG_LAUNCH = 128, REG_CTRL = 72, REG_REC = 168, REG_ENG = 104;
static_assert(128 * REG_CTRL + 256 * REG_REC + 128 * REG_ENG <= NTHREAD * REG_LAUNCH, "register split exceeds the launch");
constexpr unsigned SLICE_A = BM * KC;
constexpr unsigned SLICE_B = BN * KC;
constexpr int SMEM_AVAIL = 227 * 1024 - 2048;
constexpr unsigned long long WAIT_LIMIT_NS = 4000000000ull;

// fused energies: the f tiles of one tile pair (both orientations, 8 planes of 16 x 16 doubles each)
constexpr unsigned PARK_BYTES = 2u * 8u * 16u * 16u * 8u;

template <int S>
struct Cfg {
    static constexpr unsigned STAGE = S * (SLICE_A + SLICE_B);
    static constexpr int FIT = (SMEM_AVAIL - (int)PARK_BYTES) / (int)STAGE;
    static constexpr int STAGES = FIT > 4 ? 4 : FIT;
    static constexpr size_t SMEM = (size_t)STAGES * STAGE + PARK_BYTES + 1024;  // stages, then the park
    static constexpr unsigned TMEM_COLS = S * BN <= 256 ? 256u : 512u;
    static_assert(STAGES >= 2, "fewer than two stages fit");
    static_assert(S * BN <= 512, "level accumulators exceed tensor memory");
};

// instruction descriptor, kind::i8: D s32 (bits 4-5 = 2), A and B signed (bits 7-9, 10-12 = 1),
// both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr unsigned IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(BN >> 3) << 17) |
                           ((unsigned)(BM >> 4) << 24);

struct GemmParams {
    CUtensorMap mapA, mapB;  // 64-byte aligned members first
    CUtensorMap fmap;        // fused energies: efbuf as {V rows (contiguous), V columns, 8 * enpos planes}
    trpdrv_dev_system sys;   // fused energies: vectors, triples and energy slots of the system
    const double *ea, *eb;   // power-of-two scales per A row / B column
    const int32_t *triples, *order;
    long long pos0, ntriples, nt;  // ntriples records = n_a * nt triples per a
    double *fbuf;            // [batch][8][V][V]
    // fused energies: the energies of positions epos0 .. epos0 + enpos - 1, whose f an earlier launch
    // stored (at the fmap's base); unit u = tile pair u % np of position epos0 + u / np
    long long epos0;
    int enpos, np;
    int V, O, nks, mtiles, ntiles, tiles;  // tiles = 2 * npos * mtiles * ntiles
    int *status;
};

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

// Bounded wait; false (and status bit 1) when it runs out.
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity, int *status)
{
    if (mbar_try_wait(b, parity)) return true;
    const unsigned long long t0 = globaltimer();
    for (;;) {
#pragma unroll 1
        for (int spin = 0; spin < 256; ++spin)
            if (mbar_try_wait(b, parity)) return true;
        if (globaltimer() - t0 > WAIT_LIMIT_NS) {
            atomicOr(status, 2);
            return false;
        }
    }
}

// L2 cache policies for loads and stores: evict_last for data read again soon (the digit planes, reused
// across the tiles and triples that share them), evict_first for data read once
__device__ __forceinline__ unsigned long long policy_evict_last()
{
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ unsigned long long policy_evict_first()
{
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ void tma_load_3d_hint(void *dst, const CUtensorMap *map, unsigned long long *bar, int x,
                                                 int y, int z, unsigned long long pol)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%3, "
        "%4, %5}], [%2], %6;" ::"r"(saddr(dst)),
        "l"(map), "r"(saddr(bar)), "r"(x), "r"(y), "r"(z), "l"(pol)
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(unsigned *dst, unsigned ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(dst)), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major operand tile in shared memory with the 64-byte swizzle: rows of 64 bytes, 8-row atoms of
// 512 bytes (stride byte offset 512), leading byte offset unused (1), descriptor version 1.
__device__ __forceinline__ unsigned long long sdesc_sw64(const void *p)
{
    const unsigned a = saddr(p);
    return (unsigned long long)((a >> 4) & 0x3FFFu) | (1ull << 16) | ((unsigned long long)(512 >> 4) << 32) |
           (1ull << 46) | (4ull << 61);
}

// A-operand collector buffer use of one MMA: the first MMA of a run that shares its A tile fills the
// buffer, the following ones read A from it instead of shared memory, the last one releases it.
enum { COL_DISCARD = 0, COL_FILL = 1, COL_USE = 2, COL_LASTUSE = 3 };

__device__ __forceinline__ void mma_i8(unsigned d, unsigned long long a, unsigned long long b, int accumulate,
                                       int col = COL_DISCARD)
{
#define OZ_MMA_I8(Q)                                                                                          \
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"                                                 \
                 " tcgen05.mma.cta_group::1.kind::i8" Q " [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d), \
                 "l"(a), "l"(b), "r"(IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)                 \
                 : "memory")
    if (col == COL_FILL)
        OZ_MMA_I8(".collector::a::fill");
    else if (col == COL_USE)
        OZ_MMA_I8(".collector::a::use");
    else if (col == COL_LASTUSE)
        OZ_MMA_I8(".collector::a::lastuse");
    else
        OZ_MMA_I8("");
#undef OZ_MMA_I8
}

// collector use of the q-th of n MMAs in a row that share one A tile
__host__ __device__ constexpr int collector_op(int q, int n)
{
    return n == 1 ? COL_DISCARD : q == 0 ? COL_FILL : q == n - 1 ? COL_LASTUSE : COL_USE;
}

__device__ __forceinline__ void mma_commit(unsigned long long *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

// 32 lanes x 16 columns of 32 bits into v (valid only after tmem_wait_ld and reg_fence16)
__device__ __forceinline__ void tmem_ld16_nowait(unsigned taddr, unsigned (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Orders every use of v after the preceding tcgen05.wait::ld (volatile asm keeps its place in
// program order, and the registers pass through it).
__device__ __forceinline__ void reg_fence16(unsigned (&v)[16])
{
    asm volatile(""
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                   "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                   "+r"(v[15]));
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *b)
{
    asm volatile("mbarrier.arrive.shared.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
}

// weight of level L (0-based, slices p + q = L + 2 in 1-based digits): 2^(-7 (L + 2)), exact
__device__ __forceinline__ double level_weight(int L)
{
    double w = 1.0 / 16384.0;
    for (int l = 0; l < L; ++l) w *= 1.0 / 128.0;
    return w;
}

// ------------------------------------------------------------------------------------------------
constexpr int TW = 16;
constexpr size_t TSMEM_BYTES = (size_t)16 * TW * (TW + 1) * sizeof(double);
// TMA form (even nvir): the eight f tiles of one orientation arrive as one 16 x 16 x 8 box with the
// 128-byte swizzle; both orientations take 32 KB on a 1024-byte boundary.
constexpr int TBOX = TW * TW * 8;  // doubles of one orientation
constexpr size_t TSMEM_TMA_BYTES = (size_t)2 * TBOX * sizeof(double) + 1024;
// The plans launch 128-thread CTAs (at most 96 registers, five per SM); 256 is the other size the
// launcher accepts.  The energies of one batch are launched on a second stream after its contraction
// launch; since the contraction kernel holds every register of its SMs (512 threads x 128), they run
// on the SMs it has left, between its launches.


struct TengyItem {
    int i, j, k, pairi, y, b0, c0;
    bool diag;
    unsigned ai;
    long long tt;
};

// Geometry of work item (16-wide tile pair, batch position y after pos0), from indices alone; false for
// positions past the end of the system.
__device__ __forceinline__ bool tengy_geom(const trpdrv_dev_system &S, long long pos0, int pairi, int y,
                                           TengyItem &it)
{
    if (pos0 + y >= S.ntriples || S.nt <= 0) return false;
    const int nb = (S.nvir + TW - 1) / TW;
    int B = 0, rem = pairi;
    while (B < nb && rem >= nb - B) {
        rem -= nb - B;
        ++B;
    }
    it.pairi = pairi;
    it.y = y;
    it.b0 = B * TW;
    it.c0 = (B + rem) * TW;
    it.diag = rem == 0;
    return true;
}

// The item's triple (its record and indices); false for a malformed queue entry.
__device__ __forceinline__ bool tengy_triple(const trpdrv_dev_system &S, long long pos0, TengyItem &it)
{
    const long long pos = pos0 + it.y;  // a position over the records ([a][triple])
    it.ai = pos >= S.nt ? (unsigned)pos / (unsigned)S.nt : 0u;  // records < 2^31
    const long long tpos = pos - (long long)it.ai * S.nt;
    it.tt = S.order ? (long long)S.order[tpos] : tpos;
    if (it.tt < 0 || it.tt >= S.nt) return false;
    const int packed = S.triples[it.tt];
    it.i = packed & 1023;
    it.j = (packed >> 10) & 1023;
    it.k = (packed >> 20) & 1023;
    return true;
}

__device__ __forceinline__ bool tengy_decode(const trpdrv_dev_system &S, long long pos0, int pairi, int y,
                                             TengyItem &it)
{
    return tengy_geom(S, pos0, pairi, y, it) && tengy_triple(S, pos0, it);
}

// The vectors and eaijk of an item's triple.
__device__ __forceinline__ TengyVecs tengy_vecs(const trpdrv_dev_system &S, const TengyItem &it)
{
    const int nvir = S.nvir;
    TengyVecs v;
    v.eorb = S.eorb;
    const size_t ao = (size_t)it.ai * S.nocc;  // the a block of the a-dependent vectors
    v.dintc1 = S.dintc + (ao + it.i) * nvir;
    v.dintx1 = S.dintx + (ao + it.i) * nvir;
    v.t1v1 = S.t1v + (ao + it.i) * nvir;
    v.dintc2 = S.dintc + (ao + it.k) * nvir;
    v.dintx2 = S.dintx + (ao + it.k) * nvir;
    v.t1v2 = S.t1v + (ao + it.k) * nvir;
    v.voff = S.ncor + S.nocc;
    v.nvir = nvir;
    // omp/ccsd_trpdrv_omp_cbody.c:126 (a is 1-based, i/j/k here 0-based)
    v.eaijk = S.eorb[S.a - 1 + it.ai] - (S.eorb[S.ncor + it.i] + S.eorb[S.ncor + it.j] + S.eorb[S.ncor + it.k]);
    return v;
}

// The per-index vectors of an item in shared memory, rows of 16: t1v(i), t1v(k), dintx(i), dintx(k),
// dintc(i), dintc(k), e_virt at b0 + r (rows 0 .. 6), then the same at c0 + q (rows 7 .. 13); zero
// past nvir.  Loaded by the CTA while the item's f tiles are in flight.
constexpr int TVROWS = 14;
__device__ __forceinline__ void tengy_stage_vecs(const TengyVecs &v, const TengyItem &it, double *vsh, int tid,
                                                 int nthreads)
{
    for (int idx = tid; idx < TVROWS * TW; idx += nthreads) {
        const int row = idx / TW, x = idx % TW, side = row / 7, kind = row % 7;
        const int n = (side ? it.c0 : it.b0) + x;
        const double *src = kind == 0 ? v.t1v1 : kind == 1 ? v.t1v2 : kind == 2 ? v.dintx1 : kind == 3 ? v.dintx2
                          : kind == 4 ? v.dintc1 : kind == 5 ? v.dintc2 : v.eorb + v.voff;
        vsh[idx] = n < v.nvir ? __ldg(src + n) : 0.0;
    }
}

// The item's four energy slots (e4i, e5i, e4k, e5k).
__device__ __forceinline__ double *tengy_slot(const trpdrv_dev_system &S, const TengyItem &it)
{
    return S.partial + ((size_t)((long long)it.ai * S.nt + it.tt) * S.npairs * TRPDRV_FUSED_SLOTS + it.pairi) * 4;
}

// number of 16-wide tile pairs (must fit in the npairs * TRPDRV_FUSED_SLOTS slots of a triple)
__host__ __device__ inline int tengy_pairs(int nvir)
{
    const int nb = (nvir + TW - 1) / TW;
    return nb * (nb + 1) / 2;
}


// ------------------------------------------------------------------------------------------------
// energies fused into the contraction kernel: once every tile of a position has stored its f, the
// recombination warps of any CTA take that position's tile pairs (units) in order and compute their
// energies from f that is still in L2, in the time the next tile's products run on the tensor cores
// ------------------------------------------------------------------------------------------------
constexpr int NENG_THREADS = 32 * NENG;

// named barrier 1 over the energy warps (barrier 0 is the CTA's)
__device__ __forceinline__ void eng_bar() { asm volatile("bar.sync 1, %0;" ::"n"(NENG_THREADS) : "memory"); }

// the energy barrier, true in every thread when p is true in any
__device__ __forceinline__ bool eng_bar_or(bool p)
{
    unsigned r;
    asm volatile("{\n .reg .pred a, b;\n setp.ne.u32 a, %1, 0;\n bar.red.or.pred b, 1, %2, a;\n selp.u32 %0, 1, 0, b;\n}\n"
                 : "=r"(r)
                 : "r"((unsigned)p), "n"(NENG_THREADS)
                 : "memory");
    return r != 0;
}

// One unit's energies, by the energy threads (te = 0 .. NENG_THREADS - 1); false if the wait for its
// tiles ran out (status bit 1 set).
__device__ __forceinline__ bool fused_unit(const GemmParams &P, int u, double *park, double *vsh,
                                           unsigned long long *ubar, unsigned &uphase, double *red, int te)
{
    TengyItem it;
    if (!tengy_geom(P.sys, P.epos0, u % P.np, u / P.np, it)) return true;  // same outcome in every thread
    // the tiles' coordinates need no loads: copies first, the triple and the vectors while they land
    if (te == 0) {
        // this park's previous reads (generic proxy) before the tensor-copy writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(ubar, (it.diag ? 1u : 2u) * (PARK_BYTES / 2u));
        const unsigned long long pol = policy_evict_first();
        tma_load_3d_hint(park, &P.fmap, ubar, it.b0, it.c0, it.y * 8, pol);
        if (!it.diag) tma_load_3d_hint(park + PARK_BYTES / 16u, &P.fmap, ubar, it.c0, it.b0, it.y * 8, pol);
    }
    const bool valid = tengy_triple(P.sys, P.epos0, it);  // the same in every thread
    TengyVecs v;
    if (valid) {
        v = tengy_vecs(P.sys, it);
        tengy_stage_vecs(v, it, vsh, te, NENG_THREADS);
    }
    const bool ok = mbar_wait(ubar, uphase, P.status);
    uphase ^= 1u;
    if (eng_bar_or(!ok)) return false;  // also: the vector table is complete
    if (!valid) {
        eng_bar();  // the park and the table are free again
        return true;
    }
    TengySums su = {0.0, 0.0, 0.0, 0.0};
    tengy_tile_pair_swz16_sv<NENG_THREADS>(park, vsh, it.b0, it.c0, it.diag, v.nvir, v.eaijk, te, su);
    su.e4i = warp_sum(su.e4i);
    su.e5i = warp_sum(su.e5i);
    su.e4k = warp_sum(su.e4k);
    su.e5k = warp_sum(su.e5k);
    const int we = te >> 5;
    if ((te & 31) == 0) {
        red[4 * we + 0] = su.e4i;
        red[4 * we + 1] = su.e5i;
        red[4 * we + 2] = su.e4k;
        red[4 * we + 3] = su.e5k;
    }
    eng_bar();  // also: every read of the park is done before the next unit's copies
    if (te == 0) {
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        for (int w = 0; w < NENG; ++w)  // fixed order: the sums do not depend on which CTA ran the unit
            for (int e = 0; e < 4; ++e) t[e] += red[4 * w + e];
        double *out = tengy_slot(P.sys, it);
        out[0] = t[0];
        out[1] = t[1];
        out[2] = t[2];
        out[3] = t[3];
    }
    return true;
}

// The energy warps' loop: CTA b takes units b, b + grid, ... of the positions whose f an earlier
// launch stored, while this launch's tiles run on the tensor cores.
__device__ __forceinline__ void fused_energies(const GemmParams &P, double *park, unsigned long long *ubar,
                                               double *red, int te)
{
    const unsigned total = (unsigned)P.enpos * (unsigned)P.np;
    __shared__ double vsh[TVROWS * TW];
    unsigned uphase = 0;
    for (unsigned u = blockIdx.x; u < total; u += gridDim.x)
        if (!fused_unit(P, (int)u, park, vsh, ubar, uphase, red, te)) return;
}

// ------------------------------------------------------------------------------------------------
// contraction kernel (persistent: CTA b takes tiles b, b + grid, ...)
// ------------------------------------------------------------------------------------------------
struct Tile {
    int ok, y, grp, planeA, planeB, m0, n0;
};

__device__ __forceinline__ Tile decode_tile(const GemmParams &P, int t)
{
    Tile d;
    const int per = P.mtiles * P.ntiles;
    d.y = t / per;
    const int rem = t - d.y * per;
    d.m0 = (rem % P.mtiles) * BM;
    d.n0 = (rem / P.mtiles) * BN;
    d.grp = d.y & 1;
    const long long pos = P.pos0 + (d.y >> 1);  // a position over the records ([a][triple])
    // records < 2^31 (the host checks): 32-bit division, none for a single a
    const unsigned ai = (P.nt > 0 && pos >= P.nt) ? (unsigned)pos / (unsigned)P.nt : 0u;
    const long long tpos = pos - (long long)ai * P.nt;
    const long long tt = (pos < P.ntriples) ? (P.order ? (long long)P.order[tpos] : tpos) : -1;
    const int packed = (tt >= 0 && tt < P.nt) ? P.triples[tt] : -1;
    const int i = packed & 1023, j = (packed >> 10) & 1023, k = (packed >> 20) & 1023;
    d.ok = packed >= 0 && i < P.O && j < P.O && k < P.O;
    d.planeA = (int)ai * P.O + (d.grp ? k : i);  // the A operands carry the a index
    d.planeB = j * P.O + (d.grp ? i : k);
    return d;
}

// level accumulators are drained in groups of up to 4: X = sum_l C_l 128^(last - l) is exact in
// int64 and below 2^53 (|C_l| < 2^24), so one exact conversion and one FMA cover the group
constexpr int LGROUP = 4;

template <int S>
__global__ void __launch_bounds__(NTHREAD, 1) oz_gemm_kernel(const __grid_constant__ GemmParams P)
{
    using C = Cfg<S>;
    extern __shared__ char smem_raw[];
    __shared__ __align__(8) unsigned long long full[C::STAGES], empty[C::STAGES], tfull[1], tempty[1], done[1], ubar[1];
    __shared__ unsigned tmem_sh;
    __shared__ double red[4 * NENG];
    char *stages = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    double *park = reinterpret_cast<double *>(stages + (size_t)C::STAGES * C::STAGE);  // 1024-byte aligned

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nchunks = (P.nks * KSTEP + KC - 1) / KC;

    if (tid == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(tfull, 1);
        mbar_init(tempty, NREC);  // one arrival per recombination warp
        mbar_init(done, 1);
        mbar_init(ubar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(&tmem_sh, C::TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_sh;

    // each role's code sits in the branch of its warpgroup's register change
    if (warp < REC0) {
      asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REG_CTRL));
      if (warp == 0) {
        if (lane == 0) {  // TMA producer: runs ahead across tiles, bounded by the stage ring
            const unsigned long long pol = policy_evict_last();
            int stage = 0;
            unsigned phase = 0;
            bool alive = true;
            for (int t = blockIdx.x; alive && t < P.tiles; t += gridDim.x) {
                const Tile d = decode_tile(P, t);
                if (!d.ok) {
                    atomicOr(P.status, 1);
                    continue;
                }
                for (int kc = 0; kc < nchunks; ++kc) {
                    if (!mbar_wait(&empty[stage], phase ^ 1, P.status)) {
                        alive = false;
                        break;
                    }
                    mbar_arrive_expect_tx(&full[stage], C::STAGE);
                    char *sA = stages + (size_t)stage * C::STAGE, *sB = sA + S * SLICE_A;
                    // the digit planes are reused by the tiles and triples that share them: evict_last
#pragma unroll
                    for (int p = 0; p < S; ++p)
                        tma_load_3d_hint(sA + p * SLICE_A, &P.mapA, &full[stage], kc * KC, d.m0, d.planeA * S + p, pol);
#pragma unroll
                    for (int q = 0; q < S; ++q)
                        tma_load_3d_hint(sB + q * SLICE_B, &P.mapB, &full[stage], kc * KC, d.n0, d.planeB * S + q, pol);
                    if (++stage == C::STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer: level L = p + q (0-based) accumulates at columns L*BN..
            int stage = 0;
            unsigned phase = 0;
            bool alive = true;
            int it = 0;
            for (int t = blockIdx.x; alive && t < P.tiles; t += gridDim.x, ++it) {
                const Tile d = decode_tile(P, t);
                // the accumulators are free once the previous tile has been drained
                if (!mbar_wait(tempty, (it & 1) ^ 1, P.status)) break;
                tc_fence_after();
                if (d.ok) {
                    for (int kc = 0; kc < nchunks; ++kc) {
                        if (!mbar_wait(&full[stage], phase, P.status)) {
                            alive = false;
                            break;
                        }
                        tc_fence_after();
                        const char *sA = stages + (size_t)stage * C::STAGE, *sB = sA + S * SLICE_A;
                        const unsigned long long dA = sdesc_sw64(sA), dB = sdesc_sw64(sB);
#pragma unroll
                        for (int ks = 0; ks < KC / KSTEP; ++ks) {
                            const int kg = kc * (KC / KSTEP) + ks;
                            if (kg < P.nks) {
#pragma unroll
                                for (int p = 0; p < S; ++p)
#pragma unroll
                                    for (int q = 0; p + q < S; ++q)  // S - p MMAs share A slice p
                                        mma_i8(tmem + (unsigned)((p + q) * BN),
                                               dA + (unsigned long long)(p * (SLICE_A >> 4) + ks * (KSTEP >> 4)),
                                               dB + (unsigned long long)(q * (SLICE_B >> 4) + ks * (KSTEP >> 4)),
                                               (kg > 0 || p > 0) ? 1 : 0, collector_op(q, S - p));
                            }
                        }
                        mma_commit(&empty[stage]);  // the stage is free once these MMAs have read it
                        if (++stage == C::STAGES) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                }
                mma_commit(tfull);  // this tile's sums are complete (or the tile was skipped)
            }
            if (it > 0) {  // a CTA with no tiles (an energies-only launch) issued nothing to wait for
                mma_commit(done);  // every MMA issued by this thread has completed when `done` flips
                mbar_wait(done, 0, P.status);
            }
        }
        __syncwarp();
      }
    } else if (warp < ENG0) {  // recombination: TMEM lanes 32*(warp%4).., columns 32*half..
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(REG_REC));
        const int qd = warp & 3, half = (warp - REC0) >> 2;
        constexpr int WC = BN / 2;  // columns per recombination warp
        const int V = P.V;
        const size_t vv = (size_t)V * V;
        int it = 0;
        for (int t = blockIdx.x; t < P.tiles; t += gridDim.x, ++it) {
            const Tile d = decode_tile(P, t);
            if (!mbar_wait(tfull, it & 1, P.status)) break;
            tc_fence_after();
            double acc[WC];
#pragma unroll
            for (int c = 0; c < WC; ++c) acc[c] = 0.0;
            if (d.ok) {
                const unsigned base = tmem + ((unsigned)(qd * 32) << 16) + (unsigned)(half * WC);
#pragma unroll
                for (int cb = 0; cb < WC / 16; ++cb) {
#pragma unroll
                    for (int g0 = 0; g0 < S; g0 += LGROUP) {
                        const int g1 = (g0 + LGROUP < S) ? g0 + LGROUP : S;  // levels g0..g1-1
                        unsigned v[LGROUP][16];
#pragma unroll
                        for (int l = 0; l < LGROUP; ++l)
                            if (g0 + l < g1) tmem_ld16_nowait(base + (unsigned)((g0 + l) * BN + cb * 16), v[l]);
                        tmem_wait_ld();
#pragma unroll
                        for (int l = 0; l < LGROUP; ++l)
                            if (g0 + l < g1) reg_fence16(v[l]);
                        // weight of the group's last level: 2^(-7 (g1 - 1 + 2))
                        const double w = level_weight(g1 - 1);
#pragma unroll
                        for (int u = 0; u < 16; ++u) {
                            long long x = 0;
#pragma unroll
                            for (int l = 0; l < LGROUP; ++l)
                                if (g0 + l < g1) x = x * 128 + (long long)(int)v[l][u];
                            acc[cb * 16 + u] = fma((double)x, w, acc[cb * 16 + u]);
                        }
                    }
                }
            }
            // the accumulators may be overwritten by the next tile from here on
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty);
            const int r = d.m0 + qd * 32 + lane;
            if (d.ok && r < 2 * V) {
                const double sa = P.ea[(size_t)d.planeA * 2 * V + r];
                const int rh = r >= V ? 1 : 0, b = r - rh * V;
                double *fj = P.fbuf + (size_t)(d.y >> 1) * 8 * vv + (size_t)d.grp * 4 * vv;
                const double *eb = P.eb + (size_t)d.planeB * 2 * V;
#pragma unroll
                for (int c = 0; c < WC; ++c) {
                    const int col = d.n0 + half * WC + c;
                    if (col < 2 * V) {
                        const int ch = col >= V ? 1 : 0, cc = col - ch * V;
                        double *dst = fj + (size_t)(rh + 2 * ch) * vv + b + (size_t)cc * V;
                        const double val = acc[c] * sa * __ldg(eb + col);
                        __stcs(dst, val);  // evict-first: read once, by a later launch; keeps the digits in L2
                    }
                }
            }
        }
    } else {  // energy warps: the units of the positions an earlier launch stored
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REG_ENG));
        if (P.enpos > 0) fused_energies(P, park, ubar, red, tid - 32 * ENG0);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, C::TMEM_COLS);
    }
}

// ------------------------------------------------------------------------------------------------
// slicing: power-of-two scale per row and S base-128 digits per element
// ------------------------------------------------------------------------------------------------
struct SliceParams {
    const double *t2, *jvv, *kvv, *ntov, *nxov, *jov, *kov;
    signed char *out;  // [planes][S][2V][dp]
    double *scale;     // [planes][2V]
    int V, O, S, dp;
};

// One element of row r of plane `plane`; A side (SIDE 0) or B side (SIDE 1).
template <int SIDE>
__device__ __forceinline__ double slice_src(const SliceParams &P, int plane, int r, int d)
{
    const int V = P.V, O = P.O;
    const int h = r >= V ? 1 : 0, x = r - h * V;
    const size_t vv = (size_t)V * V, ov = (size_t)O * V;
    if (SIDE == 0) {
        if (d < V) return (h ? P.kvv : P.jvv)[plane * vv + x + (size_t)d * V];
        return (h ? P.nxov : P.ntov)[(size_t)(plane % O) * ov + x + (size_t)(d - V) * V];  // shared over a
    }
    if (d < V) return h ? P.t2[plane * vv + d + (size_t)x * V] : P.t2[plane * vv + x + (size_t)d * V];
    return (h ? P.jov : P.kov)[plane * ov + (d - V) + (size_t)x * O];
}

// whether row index is the contiguous one in memory for this tile (coalescing only)
template <int SIDE>
__device__ __forceinline__ bool slice_rows_contiguous(const SliceParams &P, int r0, int d0)
{
    if (SIDE == 0) return true;
    return r0 < P.V && d0 < P.V;
}

template <int SIDE>
__device__ __forceinline__ void slice_load(const SliceParams &P, int plane, int r0, int d0, double (*tile)[33],
                                           int tid)
{
    const int D = P.V + P.O, R = 2 * P.V;
    const bool rc = slice_rows_contiguous<SIDE>(P, r0, d0);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int idx = tid + 256 * e;
        const int rr = rc ? (idx & 31) : (idx >> 5), dd = rc ? (idx >> 5) : (idx & 31);
        const int r = r0 + rr, d = d0 + dd;
        tile[rr][dd] = (r < R && d < D) ? slice_src<SIDE>(P, plane, r, d) : 0.0;
    }
}

template <int SIDE>
__global__ void __launch_bounds__(256) oz_slice_kernel(const SliceParams P)
{
    __shared__ double tile[32][33];
    const int tid = threadIdx.x, row = tid >> 3, part = tid & 7;
    const int plane = blockIdx.y, r0 = blockIdx.x * 32;
    const int D = P.V + P.O, R = 2 * P.V;

    double mx = 0.0;
    for (int d0 = 0; d0 < D; d0 += 32) {
        slice_load<SIDE>(P, plane, r0, d0, tile, tid);
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) mx = fmax(mx, fabs(tile[row][part * 4 + u]));
        __syncthreads();
    }
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
    int e = 0;
    if (mx > 0.0) {
        frexp(mx, &e);  // mx = m 2^e, m in [1/2, 1)
        e += 1;         // mx 2^-e in [1/4, 1/2)
    }
    const double inv = ldexp(1.0, -e);
    const int r = r0 + row;
    if (part == 0 && r < R) P.scale[(size_t)plane * R + r] = ldexp(1.0, e);

    for (int d0 = 0; d0 < P.dp; d0 += 32) {
        slice_load<SIDE>(P, plane, r0, d0, tile, tid);
        __syncthreads();
        unsigned w[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            double x = tile[row][part * 4 + u] * inv;  // exact: power-of-two scaling
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                if (p < P.S) {
                    const double t = x * 128.0;
                    const double dg = rint(t);  // |dg| <= 64 since |x| <= 1/2
                    x = t - dg;                 // exact, |x| <= 1/2
                    w[p] |= ((unsigned)(int)dg & 0xffu) << (8 * u);
                }
            }
        }
        if (r < R) {
#pragma unroll
            for (int p = 0; p < 8; ++p)
                if (p < P.S)
                    *reinterpret_cast<unsigned *>(P.out + (((size_t)plane * P.S + p) * R + r) * P.dp + d0 + part * 4) =
                        w[p];
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------------
// batched tengy over the f of a batch: one CTA per (16-wide tile pair, triple), six or more CTAs per
// SM.  A CTA's four sums go to its own slot of the triple's items (slot index = tile-pair index; the
// 16-wide pairs fit in the 8 slots of each 32-wide item, and the slots no CTA writes are zero from
// plan creation), so item_reduce sums them in a fixed order.
struct TengyParams {
    CUtensorMap fmap;  // TMA form: fbuf as {nvir rows (contiguous), nvir columns, 8 * npos planes}
    trpdrv_dev_system sys;
    long long pos0;
    const double *fbuf;
    int *status;  // bit 1: a wait for the tiles ran out (the item's energies are not written)
};

// cp.async form: park f(B,C) (o = 0) and f(C,B) (o = 1) tiles of all eight f, W x (W + 1) doubles
// each; column q of a tile is contiguous in f.  Every copy of a thread is issued before any is
// waited for (zero fill outside nvir), so that a CTA keeps its whole 32 KB in flight.
template <int TNTHREAD>
__device__ __forceinline__ void tengy_park_cpasync(const TengyParams &P, const TengyItem &it, double *park)
{
    constexpr int TP = TW + 1, TILE = TW * TP;
    const int nvir = P.sys.nvir;
    const size_t lnvv = (size_t)nvir * nvir;
    const double *f = P.fbuf + (size_t)it.y * 8 * lnvv;
    const int ntiles = it.diag ? 8 : 16;
    for (int idx = threadIdx.x; idx < ntiles * TW * TW; idx += TNTHREAD) {
        const int tile = idx / (TW * TW), q = (idx / TW) % TW, r = idx % TW;
        const int o = tile >> 3, xf = tile & 7;
        const int row = (o ? it.c0 : it.b0) + r, col = (o ? it.b0 : it.c0) + q;
        const bool ok = row < nvir && col < nvir;
        cp_async_8(park + tile * TILE + r * TP + q, ok ? f + (size_t)xf * lnvv + row + (size_t)col * nvir : f, ok);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
}

// Energies of one item from its tiles parked by cp.async, summed over the CTA into its slot.
template <int TNTHREAD>
__device__ __forceinline__ void tengy_finish(const TengyParams &P, const TengyItem &it, const double *park, double *red)
{
    const int tid = threadIdx.x;
    const TengyVecs v = tengy_vecs(P.sys, it);
    TengySums su = {0.0, 0.0, 0.0, 0.0};
    tengy_tile_pair_factored<TW>(park, it.b0, it.c0, it.diag, v, tid, TNTHREAD, su);
    const TengySums tot = block_sum4(su, red);
    if (tid == 0) {  // block_sum4's result is valid in thread 0
        double *out = tengy_slot(P.sys, it);
        out[0] = tot.e4i;
        out[1] = tot.e5i;
        out[2] = tot.e4k;
        out[3] = tot.e5k;
    }
    __syncthreads();  // the park and the reduction scratch are reused by the CTA's next item
}

// CTA b takes items b, b + grid, ... (the launches use one CTA per item).
template <int TNTHREAD, bool TMA>
__global__ void __launch_bounds__(TNTHREAD, TNTHREAD == 128 ? 5 : 1)
oz_tengy_kernel(const __grid_constant__ TengyParams P, int np, int npos)
{
    extern __shared__ __align__(16) double tsmem[];
    __shared__ double red[4 * (TNTHREAD / 32)];
    __shared__ __align__(8) unsigned long long tbar[1];
    double *park = TMA ? reinterpret_cast<double *>((reinterpret_cast<uintptr_t>(tsmem) + 1023) & ~(uintptr_t)1023)
                       : tsmem;
    if (TMA) {
        if (threadIdx.x == 0) {
            mbar_init(tbar, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
    }
    unsigned phase = 0;
    const long long items = (long long)np * npos;
    for (long long w = blockIdx.x; w < items; w += gridDim.x) {
        TengyItem it;
        if (TMA) {  // the tiles' coordinates need no loads: copies first, the triple and vectors meanwhile
            __shared__ double vsh[TVROWS * TW];
            if (!tengy_geom(P.sys, P.pos0, (int)(w % np), (int)(w / np), it)) continue;  // uniform over the CTA
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive_expect_tx(tbar, (it.diag ? 1u : 2u) * (unsigned)(TBOX * sizeof(double)));
                const unsigned long long pol = policy_evict_first();
                tma_load_3d_hint(park, &P.fmap, tbar, it.b0, it.c0, it.y * 8, pol);
                if (!it.diag) tma_load_3d_hint(park + TBOX, &P.fmap, tbar, it.c0, it.b0, it.y * 8, pol);
            }
            const bool valid = tengy_triple(P.sys, P.pos0, it);  // the same in every thread
            TengyVecs v;
            if (valid) {
                v = tengy_vecs(P.sys, it);
                tengy_stage_vecs(v, it, vsh, threadIdx.x, TNTHREAD);
            }
            const bool ok = mbar_wait(tbar, phase, P.status);
            phase ^= 1;
            if (__syncthreads_or(!ok)) return;  // status bit 1 is set
            if (!valid) {
                __syncthreads();  // the park is free again
                continue;
            }
            TengySums su = {0.0, 0.0, 0.0, 0.0};
            tengy_tile_pair_swz16_sv<TNTHREAD>(park, vsh, it.b0, it.c0, it.diag, v.nvir, v.eaijk, threadIdx.x, su);
            const TengySums tot = block_sum4(su, red);
            if (threadIdx.x == 0) {
                double *out = tengy_slot(P.sys, it);
                out[0] = tot.e4i;
                out[1] = tot.e5i;
                out[2] = tot.e4k;
                out[3] = tot.e5k;
            }
            __syncthreads();  // the park, the vectors and the reduction scratch are reused by the next item
            continue;
        }
        // cp.async form (odd nvir)
        if (!tengy_decode(P.sys, P.pos0, (int)(w % np), (int)(w / np), it)) continue;  // uniform over the CTA
        tengy_park_cpasync<TNTHREAD>(P, it, park);
        tengy_finish<TNTHREAD>(P, it, park, red);
    }
}


// ------------------------------------------------------------------------------------------------
// host side
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

// 3-D map over int8 digits: dims {dp (contiguous), 2V, planes*S}, box {KC, rows, 1}, 64-byte swizzle
static int make_map_i8(CUtensorMap *m, const signed char *base, unsigned long long dp, unsigned long long rows,
                       unsigned long long planes, unsigned box_rows)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) return 1;
    const cuuint64_t dims[3] = {dp, rows, planes};
    const cuuint64_t strides[2] = {dp, dp * rows};
    const cuuint32_t box[3] = {(cuuint32_t)KC, box_rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<signed char *>(base), dims, strides, box,
                          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 2;
}

// 3-D map over the f of a batch for the TMA form of the energies: dims {nvir rows (contiguous), nvir
// columns, planes}, box {16, 16, 8} (the eight f of one triple), 128-byte swizzle, zero fill past nvir.
// Needs even nvir (row pitch a multiple of 16 bytes) and a 16-byte aligned base.
static int make_map_f64(CUtensorMap *m, const double *base, int nvir, unsigned long long planes)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || nvir < 2 || (nvir & 1) || (reinterpret_cast<uintptr_t>(base) & 15)) return 1;
    const cuuint64_t dims[3] = {(cuuint64_t)nvir, (cuuint64_t)nvir, planes};
    const cuuint64_t strides[2] = {(cuuint64_t)nvir * sizeof(double), (cuuint64_t)nvir * nvir * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)TW, (cuuint32_t)TW, 8};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 2;
}

// TRPDRV_OZ_TENGY_TMA=0 keeps the cp.async form of the energies for every nvir.
static bool tengy_tma_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("TRPDRV_OZ_TENGY_TMA");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on != 0;
}

template <int S>
static int set_attr()
{
    return (int)cudaFuncSetAttribute(oz_gemm_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)Cfg<S>::SMEM);
}

template <int S>
static int launch_gemm(const GemmParams &P, dim3 grid, cudaStream_t st)
{
    oz_gemm_kernel<S><<<grid, NTHREAD, Cfg<S>::SMEM, st>>>(P);
    return (int)cudaGetLastError();
}

}  // namespace oz
}  // namespace trpdrv

using namespace trpdrv;

// Registers per thread the contraction kernels are launched with (read back at init): the setmaxnreg
// split is valid only when every instantiation has exactly REG_LAUNCH.
static int g_oz_launch_regs = 0;

extern "C" int trpdrv_oz_slices_supported(int slices) { return slices >= TRPDRV_OZ_MIN_SLICES && slices <= TRPDRV_OZ_MAX_SLICES; }

extern "C" int trpdrv_oz_dp(int nocc, int nvir) { return ((nvir + nocc) + 31) / 32 * 32; }

// Energies inside the contraction launch (the default for even nvir: the f tiles are read by TMA): the
// kernel's energy warps compute the previous batch's energies while the tensor cores run this batch's
// products; 1.3 % faster than the separate energy launch at (40, 300), 3.4 % at (30, 400), 7 slices.
// TRPDRV_OZ_FUSED_ENERGY=0 (read at each call) selects the separate launch for every nvir.
extern "C" int trpdrv_oz_fused_energy_supported(int nvir)
{
    const char *e = getenv("TRPDRV_OZ_FUSED_ENERGY");
    const int on = !(e && e[0] == '0');
    return on && nvir >= 2 && (nvir & 1) == 0 && oz::tengy_tma_enabled();
}

extern "C" size_t trpdrv_oz_maps_bytes(void) { return 2 * sizeof(CUtensorMap); }

extern "C" int trpdrv_oz_prepare(const trpdrv_oz_system *oz, void *maps_out)
{
    CUtensorMap *m = static_cast<CUtensorMap *>(maps_out);
    const unsigned long long R = 2ull * oz->nvir, O = (unsigned long long)oz->nocc, S = (unsigned long long)oz->slices;
    const unsigned long long NA = (unsigned long long)(oz->n_a > 0 ? oz->n_a : 1);
    int e = oz::make_map_i8(&m[0], oz->sa, (unsigned long long)oz->dp, R, NA * O * S, oz::BM);
    if (e) return e;
    return oz::make_map_i8(&m[1], oz->sb, (unsigned long long)oz->dp, R, O * O * S, oz::BN);
}

extern "C" int trpdrv_launch_oz_slices(const trpdrv_dev_system *h_sys, const trpdrv_oz_system *oz, void *stream)
{
    oz::SliceParams P;
    P.t2 = h_sys->t2;
    P.jvv = h_sys->jvv;
    P.kvv = h_sys->kvv;
    P.ntov = h_sys->ntov;
    P.nxov = h_sys->nxov;
    P.jov = h_sys->jov;
    P.kov = h_sys->kov;
    P.V = oz->nvir;
    P.O = oz->nocc;
    P.S = oz->slices;
    P.dp = oz->dp;
    const unsigned rb = (unsigned)((2 * oz->nvir + 31) / 32);
    cudaStream_t st = (cudaStream_t)stream;
    P.out = oz->sa;
    P.scale = oz->ea;
    oz::oz_slice_kernel<0><<<dim3(rb, (unsigned)(oz->nocc * (oz->n_a > 0 ? oz->n_a : 1))), 256, 0, st>>>(P);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    P.out = oz->sb;
    P.scale = oz->eb;
    oz::oz_slice_kernel<1><<<dim3(rb, (unsigned)(oz->nocc * oz->nocc)), 256, 0, st>>>(P);
    return (int)cudaGetLastError();
}

extern "C" int trpdrv_launch_oz_gemm(const trpdrv_dev_system *h_sys, const trpdrv_oz_system *oz, const void *maps,
                                     int64_t pos0, int npos, double *fbuf, int64_t epos0, int enpos,
                                     const double *efbuf, int *status, int grid, void *stream)
{
    if (npos < 0 || enpos < 0 || (npos == 0 && enpos == 0)) return 0;
    oz::GemmParams P;
    memset(&P, 0, sizeof(P));
    if (enpos > 0) {  // energies of an earlier launch's positions, fused into this one
        if (!trpdrv_oz_fused_energy_supported(h_sys->nvir)) return (int)cudaErrorInvalidValue;
        P.np = oz::tengy_pairs(h_sys->nvir);
        if (P.np > h_sys->npairs * TRPDRV_FUSED_SLOTS) return (int)cudaErrorInvalidValue;
        if ((long long)P.np * enpos > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
        if (oz::make_map_f64(&P.fmap, efbuf, h_sys->nvir, 8ull * enpos) != 0) return (int)cudaErrorInvalidValue;
        P.sys = *h_sys;
        P.epos0 = epos0;
        P.enpos = enpos;
    }
    memcpy(&P.mapA, maps, sizeof(CUtensorMap));
    memcpy(&P.mapB, static_cast<const char *>(maps) + sizeof(CUtensorMap), sizeof(CUtensorMap));
    P.ea = oz->ea;
    P.eb = oz->eb;
    P.triples = h_sys->triples;
    P.order = h_sys->order;
    P.pos0 = pos0;
    P.ntriples = h_sys->ntriples;
    P.nt = h_sys->nt;
    P.fbuf = fbuf;
    P.V = oz->nvir;
    P.O = oz->nocc;
    P.nks = oz->dp / oz::KSTEP;
    P.mtiles = (2 * oz->nvir + oz::BM - 1) / oz::BM;
    P.ntiles = (2 * oz->nvir + oz::BN - 1) / oz::BN;
    P.tiles = 2 * npos * P.mtiles * P.ntiles;
    P.status = status;
    const long long work = P.tiles > 0 ? P.tiles : (long long)P.np * enpos;  // an energies-only launch
    if (grid < 1) grid = 1;
    if (grid > work) grid = (int)work;
    cudaStream_t st = (cudaStream_t)stream;
    if (g_oz_launch_regs != oz::REG_LAUNCH) return (int)cudaErrorInvalidConfiguration;  // split unusable
    switch (oz->slices) {
    case 4: return oz::launch_gemm<4>(P, dim3((unsigned)grid), st);
    case 5: return oz::launch_gemm<5>(P, dim3((unsigned)grid), st);
    case 6: return oz::launch_gemm<6>(P, dim3((unsigned)grid), st);
    case 7: return oz::launch_gemm<7>(P, dim3((unsigned)grid), st);
    case 8: return oz::launch_gemm<8>(P, dim3((unsigned)grid), st);
    default: return (int)cudaErrorInvalidValue;
    }
}

extern "C" int trpdrv_launch_oz_tengy(const trpdrv_dev_system *h_sys, int64_t pos0, int npos, const double *fbuf,
                                      int threads, int *status, void *stream)
{
    if (npos <= 0) return 0;
    const int np = oz::tengy_pairs(h_sys->nvir);
    if (np > h_sys->npairs * TRPDRV_FUSED_SLOTS) return (int)cudaErrorInvalidValue;
    if (threads != 128 && threads != 256) return (int)cudaErrorInvalidValue;
    const long long items = (long long)np * npos;
    if (items > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
    oz::TengyParams P;
    memset(&P, 0, sizeof(P));
    P.sys = *h_sys;
    P.pos0 = pos0;
    P.fbuf = fbuf;
    P.status = status;
    const bool tma = oz::tengy_tma_enabled() && oz::make_map_f64(&P.fmap, fbuf, h_sys->nvir, 8ull * npos) == 0;
    // one CTA per item: a launch of one CTA per SM (each CTA looping
    // over many items) was measured 30 % slower overall, too little memory parallelism per SM
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned grid = (unsigned)items;
    if (tma && threads == 128)
        oz::oz_tengy_kernel<128, true><<<grid, 128, oz::TSMEM_TMA_BYTES, st>>>(P, np, npos);
    else if (tma)
        oz::oz_tengy_kernel<256, true><<<grid, 256, oz::TSMEM_TMA_BYTES, st>>>(P, np, npos);
    else if (threads == 128)
        oz::oz_tengy_kernel<128, false><<<grid, 128, oz::TSMEM_BYTES, st>>>(P, np, npos);
    else
        oz::oz_tengy_kernel<256, false><<<grid, 256, oz::TSMEM_BYTES, st>>>(P, np, npos);
    return (int)cudaGetLastError();
}

template <int S>
static int oz_regs(int *all_equal)
{
    cudaFuncAttributes a;
    const cudaError_t e = cudaFuncGetAttributes(&a, oz::oz_gemm_kernel<S>);
    if (e != cudaSuccess) return (int)e;
    if (a.numRegs != oz::REG_LAUNCH) *all_equal = 0;
    return 0;
}

extern "C" int trpdrv_oz_init(void)
{
    int e, regs_ok = 1;
    if ((e = oz_regs<4>(&regs_ok)) != 0 || (e = oz_regs<5>(&regs_ok)) != 0 || (e = oz_regs<6>(&regs_ok)) != 0 ||
        (e = oz_regs<7>(&regs_ok)) != 0 || (e = oz_regs<8>(&regs_ok)) != 0)
        return e;
    g_oz_launch_regs = regs_ok ? oz::REG_LAUNCH : 0;
    if ((e = oz::set_attr<4>()) != 0) return e;
    if ((e = oz::set_attr<5>()) != 0) return e;
    if ((e = oz::set_attr<6>()) != 0) return e;
    if ((e = oz::set_attr<7>()) != 0) return e;
    if ((e = oz::set_attr<8>()) != 0) return e;
    const cudaFuncAttribute dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if ((e = (int)cudaFuncSetAttribute(oz::oz_tengy_kernel<128, false>, dyn, (int)oz::TSMEM_BYTES)) != 0) return e;
    if ((e = (int)cudaFuncSetAttribute(oz::oz_tengy_kernel<256, false>, dyn, (int)oz::TSMEM_BYTES)) != 0) return e;
    if ((e = (int)cudaFuncSetAttribute(oz::oz_tengy_kernel<128, true>, dyn, (int)oz::TSMEM_TMA_BYTES)) != 0) return e;
    return (int)cudaFuncSetAttribute(oz::oz_tengy_kernel<256, true>, dyn, (int)oz::TSMEM_TMA_BYTES);
}
