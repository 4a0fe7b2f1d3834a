// The tengy reduction over one tile pair {B,C} whose f tiles are parked in shared memory.
// Layout of `park`: 16 tiles of 32 x 33 doubles; tile (o*8 + x) holds f_x(B+r, C+q) for o = 0 and
// f_x(C+r, B+q) for o = 1 at [r*33 + q] (x = f1n f2n f3n f4n f1t f2t f3t f4t).  For a diagonal pair
// (B == C) only the o = 0 tiles are used.  Follows omp/ccsd_tengy_c99.c:58-111: every (b,c) of
// BxC and CxB contributes one term with denom = -1/(e_b + e_c + eaijk).
#pragma once

#include "device_common.cuh"

namespace trpdrv {

constexpr int TT = 32;           // tile width
constexpr int TPP = TT + 1;      // parked tile pitch
constexpr int TPTILE = TT * TPP;

struct TengyVecs {
    const double *eorb, *dintc1, *dintx1, *t1v1, *dintc2, *dintx2, *t1v2;
    double eaijk;
    int voff;  // ncor + nocc: index of the first virtual orbital energy
    int nvir;
};

// Tengy terms of one tile pair {B, C} of width W from tiles parked in shared memory: park holds the
// eight f tiles of orientation (B, C) followed (off the diagonal) by the eight of (C, B), each tile
// W x (W + 1) doubles, element (row r, column q) at r * (W + 1) + q.
template <int W>
__device__ __forceinline__ void tengy_tile_pair_w(const double *park, int b0, int c0, bool diag, const TengyVecs &v,
                                                  int tid, int nthreads, TengySums &su)
{
    constexpr int P = W + 1, TILE = W * P;
    const int nterm = diag ? W * W : 2 * W * W;
    for (int idx = tid; idx < nterm; idx += nthreads) {
        const int s = idx / (W * W), r = (idx / W) % W, q = idx % W;
        const int b = (s ? c0 : b0) + r, c = (s ? b0 : c0) + q;
        if (b < v.nvir && c < v.nvir) {
            const double *bcT = park + (s * 8) * TILE + r * P + q;
            const double *cbT = park + ((diag ? 0 : 1 - s) * 8) * TILE + q * P + r;
            double fbc[8], fcb[8];
#pragma unroll
            for (int f = 0; f < 8; ++f) {
                fbc[f] = bcT[f * TILE];
                fcb[f] = cbT[f * TILE];
            }
            const double denom = -1.0 / (__ldg(v.eorb + v.voff + b) + __ldg(v.eorb + v.voff + c) + v.eaijk);
            tengy_term(fbc, fcb, denom, __ldg(v.t1v1 + b), __ldg(v.t1v2 + b), __ldg(v.dintx1 + c),
                       __ldg(v.dintx2 + c), __ldg(v.dintc1 + c), __ldg(v.dintc2 + c), su);
        }
    }
}

// The same sums with one thread per (b, c) of B x C: the 16 values at (b, c) and (c, b) are loaded
// once, the denominator (equal for both) is formed once, and the factored forms give the terms of
// (b, c) and, off the diagonal, of (c, b).  Equal to tengy_tile_pair_w up to reassociation.
template <int W>
__device__ __forceinline__ void tengy_tile_pair_factored(const double *park, int b0, int c0, bool diag,
                                                         const TengyVecs &v, int tid, int nthreads, TengySums &su)
{
    constexpr int P = W + 1, TILE = W * P;
    for (int idx = tid; idx < W * W; idx += nthreads) {
        const int r = idx / W, q = idx % W;
        const int b = b0 + r, c = c0 + q;
        if (b < v.nvir && c < v.nvir) {
            const double *bcT = park + r * P + q;                          // f_x(B + r, C + q)
            const double *cbT = park + (diag ? 0 : 8) * TILE + q * P + r;  // f_x(C + q, B + r)
            double fbc[8], fcb[8];
#pragma unroll
            for (int f = 0; f < 8; ++f) {
                fbc[f] = bcT[f * TILE];
                fcb[f] = cbT[f * TILE];
            }
            const double denom = -1.0 / (__ldg(v.eorb + v.voff + b) + __ldg(v.eorb + v.voff + c) + v.eaijk);
            tengy_term_factored(fbc, fcb, denom, __ldg(v.t1v1 + b), __ldg(v.t1v2 + b), __ldg(v.dintx1 + c),
                                __ldg(v.dintx2 + c), __ldg(v.dintc1 + c), __ldg(v.dintc2 + c), su);
            if (!diag)
                tengy_term_factored(fcb, fbc, denom, __ldg(v.t1v1 + c), __ldg(v.t1v2 + c), __ldg(v.dintx1 + b),
                                    __ldg(v.dintx2 + b), __ldg(v.dintc1 + b), __ldg(v.dintc2 + b), su);
        }
    }
}

// Element x of the 16-double row `col` in a box landed with the 128-byte swizzle: the 16-byte chunk
// index is XORed with col mod 8 (rows are 128 bytes, the box starts on a 1024-byte boundary).
__device__ __forceinline__ int swz128(int x, int col) { return (((x >> 1) ^ (col & 7)) << 1) | (x & 1); }

// The same sums over 16-wide tiles as TMA lands them: the (B, C) box, then off the diagonal the
// (C, B) box, each 8 planes (one per f) of 16 columns x 16 rows, row index contiguous and swizzled
// by swz128.  Each half-warp walks one diagonal q = (r + d) mod 16: both the (b, c) reads (row r of
// column q) and the (c, b) reads (row q of column r) then hit 16 different 8-byte bank pairs.
template <int NTHREAD>
__device__ __forceinline__ void tengy_tile_pair_swz16(const double *park, int b0, int c0, bool diag,
                                                      const TengyVecs &v, int tid, TengySums &su)
{
    constexpr int PLANE = 16 * 16, BOX = 8 * PLANE, NDIAG = 16 / (NTHREAD / 16);
    static_assert(NTHREAD % 16 == 0 && NTHREAD <= 256 && 16 % (NTHREAD / 16) == 0, "half-warps walk the 16 diagonals");
    const int r = tid & 15;
#pragma unroll
    for (int k = 0; k < NDIAG; ++k) {  // a fixed trip count: the loads of every diagonal issue together
        const int d = (tid >> 4) + k * (NTHREAD / 16);
        const int q = (r + d) & 15;
        const int b = b0 + r, c = c0 + q;
        if (b < v.nvir && c < v.nvir) {
            const double *bcT = park + q * 16 + swz128(r, q);                       // f_x(B + r, C + q)
            const double *cbT = park + (diag ? 0 : BOX) + r * 16 + swz128(q, r);    // f_x(C + q, B + r)
            double fbc[8], fcb[8];
#pragma unroll
            for (int f = 0; f < 8; ++f) {
                fbc[f] = bcT[f * PLANE];
                fcb[f] = cbT[f * PLANE];
            }
            const double denom = -1.0 / (__ldg(v.eorb + v.voff + b) + __ldg(v.eorb + v.voff + c) + v.eaijk);
            tengy_term_factored(fbc, fcb, denom, __ldg(v.t1v1 + b), __ldg(v.t1v2 + b), __ldg(v.dintx1 + c),
                                __ldg(v.dintx2 + c), __ldg(v.dintc1 + c), __ldg(v.dintc2 + c), su);
            if (!diag)
                tengy_term_factored(fcb, fbc, denom, __ldg(v.t1v1 + c), __ldg(v.t1v2 + c), __ldg(v.dintx1 + b),
                                    __ldg(v.dintx2 + b), __ldg(v.dintc1 + b), __ldg(v.dintc2 + b), su);
        }
    }
}

// tengy_tile_pair_swz16 with the per-index vectors read from a shared table (rows of 16: t1v(i),
// t1v(k), dintx(i), dintx(k), dintc(i), dintc(k), e_virt at b0 + r, then the same seven at c0 + q).
template <int NTHREAD>
__device__ __forceinline__ void tengy_tile_pair_swz16_sv(const double *park, const double *vsh, int b0, int c0,
                                                         bool diag, int nvir, double eaijk, int tid, TengySums &su)
{
    constexpr int PLANE = 16 * 16, BOX = 8 * PLANE, NDIAG = 16 / (NTHREAD / 16);
    static_assert(NTHREAD % 16 == 0 && NTHREAD <= 256 && 16 % (NTHREAD / 16) == 0, "half-warps walk the 16 diagonals");
    const int r = tid & 15;
    const double *vb = vsh, *vc = vsh + 7 * 16;  // row x of a side at [x * 16 + index]
#pragma unroll
    for (int k = 0; k < NDIAG; ++k) {
        const int d = (tid >> 4) + k * (NTHREAD / 16);
        const int q = (r + d) & 15;
        if (b0 + r < nvir && c0 + q < nvir) {
            const double *bcT = park + q * 16 + swz128(r, q);                       // f_x(B + r, C + q)
            const double *cbT = park + (diag ? 0 : BOX) + r * 16 + swz128(q, r);    // f_x(C + q, B + r)
            double fbc[8], fcb[8];
#pragma unroll
            for (int f = 0; f < 8; ++f) {
                fbc[f] = bcT[f * PLANE];
                fcb[f] = cbT[f * PLANE];
            }
            const double denom = -1.0 / (vb[6 * 16 + r] + vc[6 * 16 + q] + eaijk);
            tengy_term_factored(fbc, fcb, denom, vb[0 * 16 + r], vb[1 * 16 + r], vc[2 * 16 + q], vc[3 * 16 + q],
                                vc[4 * 16 + q], vc[5 * 16 + q], su);
            if (!diag)
                tengy_term_factored(fcb, fbc, denom, vc[0 * 16 + q], vc[1 * 16 + q], vb[2 * 16 + r], vb[3 * 16 + r],
                                    vb[4 * 16 + r], vb[5 * 16 + r], su);
        }
    }
}

__device__ __forceinline__ void tengy_tile_pair(const double *park, int b0, int c0, bool diag,
                                                const TengyVecs &v, int tid, int nthreads, TengySums &su)
{
    tengy_tile_pair_w<TT>(park, b0, c0, diag, v, tid, nthreads, su);
}

}  // namespace trpdrv
