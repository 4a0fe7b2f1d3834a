/*
 * Internal interface between the C host layer (host.c) and the CUDA translation units.
 * Plain C structs and extern "C" launchers only; every launcher enqueues on the given stream and
 * returns a cudaError_t value (0 = success).
 */
#ifndef TRPDRV_LAUNCH_H
#define TRPDRV_LAUNCH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Width of the (b,c) tiles of the fused kernel and of the standalone tengy kernel. */
#define TRPDRV_TILE 32
/* Energy slots per fused work item (one per warp of the fused CTA). */
#define TRPDRV_FUSED_SLOTS 8
/* Triples are packed as (i-1) | (j-1) << 10 | (k-1) << 20 (0-based), so nocc must be < 1024. */
#define TRPDRV_MAX_NOCC 1023
/* Largest nvir the kernels accept (index arithmetic is 32-bit within one nvir x nvir block). */
#define TRPDRV_MAX_NVIR 16384

/* Device view of one system in a plan.  ntov/nxov hold -tov/-xov, so that every f is the sum of
 * two products accumulated with +1 (the reference's alpha = -1 GEMMs, omp/ccsd_trpdrv_omp_cbody.c:73-116). */
typedef struct trpdrv_dev_system {
    int ncor, nocc, nvir, a;
    int nb;              /* ceil(nvir / TRPDRV_TILE) */
    int npairs;          /* nb*(nb+1)/2 tile pairs (B <= C) */
    int64_t ntriples;    /* records of this system in the plan: n_a * nt */
    int64_t nt;          /* triples per a (this rank's share): the length of `triples` and `order` */
    int n_a;             /* virtual indices a .. a + n_a - 1 swept (1 = the reference driver's single a) */
    int one_triple;      /* 1: the tensors hold only what one triple (i, j, k) reads, the i-role block at
                            occupied slot 0 and the k-role block at slot 1 (t2, jov, kov: one j block
                            of two slots; jvv, kvv, ntov, nxov, dintc, dintx, t1v: two slots), as the
                            drop-in entry points stage them; `triples` holds that triple (its i, j, k
                            give eaijk) and n_a is 1.  TMA kernel only. */
    int64_t slot_stride; /* one_triple: doubles between the i-role and k-role blocks of every TMA-read tensor
                            (t2, jvv, kvv, ntov, nxov, jov, kov); 0 = the packed [2][block] layout.  The
                            vectors (dintc, dintx, t1v) stay packed [2][nvir]. */
    int split;           /* 1 (one_triple systems): every item's contraction runs as two work items (even and
                            odd chunks, item indices 2 q and 2 q + 1) on two SMs; each writes its partial f to
                            split_scratch [item][2][64][256] and the second to arrive (split_count[item])
                            adds the other's and runs the energy epilogue */
    double *split_scratch;
    unsigned *split_count;  /* one per item, zero at launch; left at zero */
    int pack_edge;       /* 1: the last tile holds 1..16 valid virtual indices and the TMA kernel runs the
                            edge pairs (B, E), (B + 1, E) (B even) as one packed work item; the item of
                            (B + 1, E) is then skipped (its energy slots are written by the packed one) */
    int64_t item_begin;  /* first fused work item of this system */
    const double *eorb, *t2, *jvv, *kvv, *ntov, *nxov, *jov, *kov, *dintc, *dintx, *t1v;
    const int32_t *triples; /* packed triples, driver order (energies are stored in this order) */
    const int32_t *order;   /* fused kernels: processing position -> triple index, or NULL (identity) */
    double *partial;        /* [ntriples*npairs][TRPDRV_FUSED_SLOTS][4]: e4i, e5i, e4k, e5k */
    double *rec;            /* [ntriples][4] per triple */
} trpdrv_dev_system;

/* Fused persistent kernel: grid CTAs pull (triple, tile pair) items from *counter (must be 0 at
 * launch) and write per-item energies.  vec2 = 1 requires even nvir and nocc for every system;
 * mma_k selects the FP64 MMA shape m16n8k4 (4) or m16n8k8 (8). */
int trpdrv_launch_fused(const trpdrv_dev_system *d_sys, int nsys, int64_t total_items,
                        unsigned long long *counter, int *status, int grid, int vec2, int mma_k,
                        void *stream);
size_t trpdrv_fused_smem_bytes(void);
int trpdrv_fused_threads(void);
int trpdrv_fused_max_ctas_per_sm(int *n);
int trpdrv_fused_init(void);

/* The same fused computation with TMA-staged panels and mbarrier pipelines (fused_tma.cu).  Needs
 * even nvir and nocc, 16-byte aligned tensors and at most TRPDRV_TMA_MAX_SYSTEMS systems
 * (trpdrv_tma_supported).  trpdrv_tma_prepare encodes the tensor maps of every system into a
 * host blob of trpdrv_tma_maps_bytes() bytes (64-byte aligned) that each launch passes by value.
 * One CTA per SM.  *status bit 0: malformed queue entry; bit 1: a pipeline wait ran out. */
#define TRPDRV_TMA_MAX_SYSTEMS 8
int trpdrv_tma_supported(const trpdrv_dev_system *h_sys, int nsys);
/* 1 if the TMA kernel packs the edge pairs of a system with this nvir (see pack_edge). */
int trpdrv_tma_pack_edge(int nvir);
size_t trpdrv_tma_maps_bytes(void);
int trpdrv_tma_prepare(const trpdrv_dev_system *h_sys, int nsys, void *maps_out);
int trpdrv_launch_fused_tma(const trpdrv_dev_system *d_sys, int nsys, int64_t total_items,
                            unsigned long long *counter, int *status, int grid, const void *maps,
                            int mma_k, int split, void *stream);
int trpdrv_fused_tma_init(void);
/* One thread waits, with the production bounded wait and the given limit, on an mbarrier that
 * nothing completes: sets bit 1 of *status when the wait gives up (bit 2 if it wrongly completes)
 * and stores how long it waited. */
int trpdrv_launch_wait_selftest(unsigned long long limit_ns, int *status, unsigned long long *elapsed_ns,
                                void *stream);

/* Emulated-FP64 (Ozaki int8) form, ozaki.cu.  Per system: digit slices of the A operands
 * sa [nocc][slices][2 nvir][dp] and of the B operands sb [nocc*nocc][slices][2 nvir][dp] (int8,
 * dp = trpdrv_oz_dp: nvir + nocc rounded up to 32), with power-of-two scales ea [nocc][2 nvir] and
 * eb [nocc*nocc][2 nvir].  trpdrv_oz_prepare encodes the two tensor maps into a host blob of
 * trpdrv_oz_maps_bytes() bytes (64-byte aligned).  A batch is npos consecutive positions of the
 * system's processing order starting at pos0: the contraction kernel writes their f into
 * fbuf [npos][8][nvir][nvir] and the tengy kernel writes the sums of each 16-wide tile pair into
 * one slot of the triple's items in `partial` (the other slots must be zero), for
 * trpdrv_launch_item_reduce.  *status as the fused kernels (bit 0 malformed entry, bit 1 a wait
 * ran out).  The contraction kernel is persistent: grid = CTAs (one per SM). */
#define TRPDRV_OZ_MIN_SLICES 4
#define TRPDRV_OZ_MAX_SLICES 8
typedef struct trpdrv_oz_system {
    int nocc, nvir, slices, dp, n_a;  /* n_a: a values swept; sa holds n_a * nocc planes */
    signed char *sa, *sb;
    double *ea, *eb;
} trpdrv_oz_system;
int trpdrv_oz_slices_supported(int slices);
int trpdrv_oz_dp(int nocc, int nvir);
size_t trpdrv_oz_maps_bytes(void);
int trpdrv_oz_prepare(const trpdrv_oz_system *oz, void *maps_out);
int trpdrv_launch_oz_slices(const trpdrv_dev_system *h_sys, const trpdrv_oz_system *oz, void *stream);
/* Products of positions pos0 .. pos0 + npos - 1 into fbuf; enpos > 0 (requires
 * trpdrv_oz_fused_energy_supported(nvir)): the same launch's energy warps also compute the energies
 * of positions epos0 .. epos0 + enpos - 1, whose f an earlier launch stored at efbuf.  npos = 0 gives an
 * energies-only launch. */
int trpdrv_launch_oz_gemm(const trpdrv_dev_system *h_sys, const trpdrv_oz_system *oz, const void *maps,
                          int64_t pos0, int npos, double *fbuf, int64_t epos0, int enpos, const double *efbuf,
                          int *status, int grid, void *stream);
int trpdrv_oz_fused_energy_supported(int nvir);
/* threads: 128 (what the plans launch) or 256.  Emulated plans launch the energies of one batch on a
 * second stream, ordered only after that batch's products.  Even nvir: the tiles
 * arrive by TMA (fbuf 16-byte aligned), with a bounded wait that sets *status bit 1 when it runs out;
 * odd nvir (or TRPDRV_OZ_TENGY_TMA=0): cp.async copies. */
int trpdrv_launch_oz_tengy(const trpdrv_dev_system *h_sys, int64_t pos0, int npos, const double *fbuf,
                           int threads, int *status, void *stream);
int trpdrv_oz_init(void);

/* Per-triple sum of the per-item energies of one system (partial -> rec). */
int trpdrv_launch_item_reduce(const trpdrv_dev_system *h_sys, void *stream);

/* Compensated per-system total over rec: out[0..3] = emp4 hi, emp4 lo, emp5 hi, emp5 lo, where the
 * total is emp4i + [i != k] emp4k summed over the triples. */
int trpdrv_launch_system_reduce(const double *rec, const int32_t *triples, int64_t ntriples, int64_t nt,
                                double *out, void *stream);

/* dst[i] = -src[i]. */
int trpdrv_launch_negate(const double *src, double *dst, size_t n, void *stream);

/* Device-to-device copies dst[s][0..len[s]) = src[s][..] (negated where neg[s]) for s < n, in one launch. */
#define TRPDRV_COPY_LIST_MAX 24
typedef struct trpdrv_copy_list {
    int n;
    const double *src[TRPDRV_COPY_LIST_MAX];
    double *dst[TRPDRV_COPY_LIST_MAX];
    long long len[TRPDRV_COPY_LIST_MAX];
    int neg[TRPDRV_COPY_LIST_MAX];  /* 1: dst = -src */
} trpdrv_copy_list;
int trpdrv_launch_gather(const trpdrv_copy_list *list, void *stream);

/* Plain per-triple path: one grouped launch computes the eight f = A1*op(B1) + A2*B2 into
 * f[8][nvir][nvir] (order f1n f2n f3n f4n f1t f2t f3t f4t); b1_nt[x] = 1 if B1 is used transposed. */
typedef struct trpdrv_plain_args {
    int nocc, nvir;
    const double *a1[8], *b1[8], *a2[8], *b2[8];
    int b1_nt[8];
    double *f;
} trpdrv_plain_args;
int trpdrv_launch_plain_gemm(const trpdrv_plain_args *args, int vec2, void *stream);

/* Standalone tengy over f[8][nvir][nvir] on the device.  eaijk is taken from `eaijk` when
 * use_eaijk != 0, else computed on the device from eorb and the 1-based a, i, j, k.  Writes
 * out4[0..3] = emp4i, emp5i, emp4k, emp5k.  block_partial needs 4*npairs doubles, counter one
 * zeroed unsigned int (it is left at zero again). */
typedef struct trpdrv_tengy_args {
    int ncor, nocc, nvir;
    int use_eaijk;
    double eaijk;
    int a, i, j, k;
    const double *f;
    const double *eorb, *dintc1, *dintx1, *t1v1, *dintc2, *dintx2, *t1v2;
    double *block_partial;
    unsigned int *counter;
    double *out4;
} trpdrv_tengy_args;
int trpdrv_launch_tengy(const trpdrv_tengy_args *args, void *stream);
size_t trpdrv_tengy_smem_bytes(void);


/* Sets the dynamic shared memory limits of every kernel (call once per device). */
int trpdrv_kernels_init(void);

/* Sets the calling thread's trpdrv_last_error() status and message; returns status. */
int trpdrv_record_error(int status, const char *message);

#ifdef __cplusplus
}
#endif
#endif
