// Device-side building blocks shared by the triples kernels (sm_100a).
//
//  * FP64 tensor-core MMA (DMMA) wrappers: mma.sync ... .f64 (sm_100a has no tcgen05 kind for
//    f64, so FP64 contractions run on the mma.sync DMMA path).
//  * cp.async global->shared staging with zero fill for masked tails.
//  * The tengy (b,c) energy term of omp/ccsd_tengy_c99.c:65-111, written once and used by both the
//    fused epilogue and the standalone reduction kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace trpdrv {

// ------------------------------------------------------------------------------------------------
// FP64 MMA.  Fragment layouts (PTX ISA, mma.m16n8k4 .f64):  g = lane>>2, t = lane&3
//   A 16x4 (row): a0 = A[g][t], a1 = A[g+8][t]
//   B 4x8  (col): b0 = B[t][g]
//   C 16x8      : c0 = C[g][2t], c1 = C[g][2t+1], c2 = C[g+8][2t], c3 = C[g+8][2t+1]
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0)
{
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a0, double b0)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a0), "d"(b0));
}

__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__device__ __forceinline__ void dmma_16x8x16(double (&d)[4], const double (&a)[8], const double (&b)[4])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
        "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
          "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// ------------------------------------------------------------------------------------------------
// cp.async staging.  `valid == false` copies nothing from global and zero-fills the destination
// (src-size operand 0); the source address is still required to be a mapped address, so callers
// pass an in-bounds base pointer in that case.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}

__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ------------------------------------------------------------------------------------------------
// Reductions
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Error-free transformation a + b = s + e (Knuth TwoSum).
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e)
{
    s = a + b;
    const double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// ------------------------------------------------------------------------------------------------
// The tengy term at one (b,c).  f index order used throughout the library:
//   0 f1n, 1 f2n, 2 f3n, 3 f4n, 4 f1t, 5 f2t, 6 f3t, 7 f4t
// bc[x] = f_x(b,c), cb[x] = f_x(c,b).  Arithmetic as omp/ccsd_tengy_c99.c:65-111.
// ------------------------------------------------------------------------------------------------
struct TengySums {
    double e4i, e5i, e4k, e5k;
};

__device__ __forceinline__ void tengy_term(const double (&bc)[8], const double (&cb)[8], double denom,
                                           double t1v1b, double t1v2b, double dx1c, double dx2c,
                                           double dc1c, double dc2c, TengySums &s)
{
    const double n1bc = bc[0], n2bc = bc[1], n3bc = bc[2], n4bc = bc[3];
    const double t1bc = bc[4], t2bc = bc[5], t3bc = bc[6], t4bc = bc[7];
    const double n1cb = cb[0], n2cb = cb[1], n3cb = cb[2], n4cb = cb[3];
    const double t1cb = cb[4], t2cb = cb[5], t3cb = cb[6], t4cb = cb[7];

    s.e4i += denom * (t1bc + n1cb + t2cb + n3bc + n4cb) * (t1bc - t2bc * 2 - t3bc * 2 + t4bc)
           - denom * (n1bc + t1cb + n2cb + n3cb) * (t1bc * 2 - t2bc - t3bc + t4bc * 2)
           + denom * 3 * (n1bc * (n1bc + n3cb + t4cb * 2) + n2bc * t2cb + n3bc * t4bc);
    s.e4k += denom * (n1bc + t1cb + n2cb + t3bc + t4cb) * (n1bc - n2bc * 2 - n3bc * 2 + n4bc)
           - denom * (t1bc + n1cb + t2cb + t3cb) * (n1bc * 2 - n2bc - n3bc + n4bc * 2)
           + denom * 3 * (t1bc * (t1bc + t3cb + n4cb * 2) + t2bc * n2cb + t3bc * n4bc);
    s.e5i += denom * t1v1b * dx1c * (t1bc + n2bc + n4cb - (t3bc + n4bc + n2cb + n1bc + t2bc + n3cb) * 2
                                     + (n3bc + t4bc + n1cb) * 4)
           + denom * t1v1b * dc1c * (n1bc + n4bc + t1cb - (n2bc + n3bc + t2cb) * 2);
    s.e5k += denom * t1v2b * dx2c * (n1bc + t2bc + t4cb - (n3bc + t4bc + t2cb + t1bc + n2bc + t3cb) * 2
                                     + (t3bc + n4bc + t1cb) * 4)
           + denom * t1v2b * dc2c * (t1bc + t4bc + n1cb - (t2bc + t3bc + n2cb) * 2);
}

// The same four forms with the denominator factored out of each, for callers that already hold
// denom = -1/(e_b + e_c + eaijk) (shared by the mirrored positions (b,c) and (c,b)).  Equal to
// tengy_term up to floating-point reassociation.
__device__ __forceinline__ void tengy_term_factored(const double (&bc)[8], const double (&cb)[8], double denom,
                                                    double t1v1b, double t1v2b, double dx1c, double dx2c,
                                                    double dc1c, double dc2c, TengySums &s)
{
    const double n1bc = bc[0], n2bc = bc[1], n3bc = bc[2], n4bc = bc[3];
    const double t1bc = bc[4], t2bc = bc[5], t3bc = bc[6], t4bc = bc[7];
    const double n1cb = cb[0], n2cb = cb[1], n3cb = cb[2], n4cb = cb[3];
    const double t1cb = cb[4], t2cb = cb[5], t3cb = cb[6], t4cb = cb[7];

    const double a4i = (t1bc + n1cb + t2cb + n3bc + n4cb) * (t1bc - t2bc * 2 - t3bc * 2 + t4bc)
                     - (n1bc + t1cb + n2cb + n3cb) * (t1bc * 2 - t2bc - t3bc + t4bc * 2)
                     + 3 * (n1bc * (n1bc + n3cb + t4cb * 2) + n2bc * t2cb + n3bc * t4bc);
    const double a4k = (n1bc + t1cb + n2cb + t3bc + t4cb) * (n1bc - n2bc * 2 - n3bc * 2 + n4bc)
                     - (t1bc + n1cb + t2cb + t3cb) * (n1bc * 2 - n2bc - n3bc + n4bc * 2)
                     + 3 * (t1bc * (t1bc + t3cb + n4cb * 2) + t2bc * n2cb + t3bc * n4bc);
    const double f5i = t1bc + n2bc + n4cb - (t3bc + n4bc + n2cb + n1bc + t2bc + n3cb) * 2 + (n3bc + t4bc + n1cb) * 4;
    const double g5i = n1bc + n4bc + t1cb - (n2bc + n3bc + t2cb) * 2;
    const double f5k = n1bc + t2bc + t4cb - (n3bc + t4bc + t2cb + t1bc + n2bc + t3cb) * 2 + (t3bc + n4bc + t1cb) * 4;
    const double g5k = t1bc + t4bc + n1cb - (t2bc + t3bc + n2cb) * 2;
    s.e4i += denom * a4i;
    s.e4k += denom * a4k;
    s.e5i += denom * (t1v1b * (dx1c * f5i + dc1c * g5i));
    s.e5k += denom * (t1v2b * (dx2c * f5k + dc2c * g5k));
}

// Block-wide sum of the four partial energies; returns the totals in thread 0.  `scratch` must
// hold 4 * (blockDim.x / 32) doubles.  The summation order is fixed (deterministic).
__device__ __forceinline__ TengySums block_sum4(TengySums s, double *scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    s.e4i = warp_sum(s.e4i);
    s.e5i = warp_sum(s.e5i);
    s.e4k = warp_sum(s.e4k);
    s.e5k = warp_sum(s.e5k);
    if (lane == 0) {
        scratch[4 * warp + 0] = s.e4i;
        scratch[4 * warp + 1] = s.e5i;
        scratch[4 * warp + 2] = s.e4k;
        scratch[4 * warp + 3] = s.e5k;
    }
    __syncthreads();
    TengySums r = {0.0, 0.0, 0.0, 0.0};
    if (threadIdx.x == 0) {
        for (int w = 0; w < nw; ++w) {
            r.e4i += scratch[4 * w + 0];
            r.e5i += scratch[4 * w + 1];
            r.e4k += scratch[4 * w + 2];
            r.e5k += scratch[4 * w + 3];
        }
    }
    return r;
}

}  // namespace trpdrv
