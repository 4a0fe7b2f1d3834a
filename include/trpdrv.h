/*
 * trpdrv.h — C ABI of the B200 (sm_100a) CCSD(T) triples-driver library, libtrpdrv_b200.so.
 *
 * Part 1 exports the reference's own entry points with the reference's exact signatures, so the
 * reference driver (omp/test.c) and Fortran/C callers link against this library unchanged.
 * Part 2 is the batched interface: whole systems (every (i,j,k) triple of one `a`, or of a range of
 * `a` with options.a_count) resident on the device, run by one persistent fused FP64 kernel, by the
 * emulated-FP64 int8 form, or by a plain per-triple path, optionally sharded over ranks.
 *
 * Conventions: all real data is IEEE double; integers are 32-bit unless typed otherwise; orbital
 * indices in the reference entry points are 1-based (Fortran convention, as in the reference).
 * Matrices are column-major: f(b,c) lives at f[b + c*nvir].  No function here takes or returns a
 * framework type; streams are passed as `void *` holding a cudaStream_t (NULL = the library's own).
 */
#ifndef TRPDRV_B200_H
#define TRPDRV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================================
 * Part 1. Reference entry points (drop-in)
 * ====================================================================================== */

/* One triple (a,i,j,k): the 16 DGEMMs forming f1n..f4t, eaijk, the tengy reduction, and
 * emp4 += emp4i (+ emp4k if i != k), emp5 likewise.
 * Replaces ccsd_trpdrv_omp_cbody_ (omp/ccsd_trpdrv_omp_cbody.c:31-44; caller prototype
 * omp/test.c:39-52).  All arguments by reference; every pointer is caller-owned HOST memory.
 * tkj, jka, kka are offset by (k-klo)*nvir*nvir and tka, xka, jkj, kkj by (k-klo)*nocc*nvir, as in
 * the reference.  f1n..f4t are scratch: they are written back only when TRPDRV_WRITE_F=1.
 * Device work per call: with even nocc and nvir (and TRPDRV_WRITE_F unset) the slices are staged
 * into a fixed one-triple layout (host slices compared with a pinned mirror and copied where they
 * differ by up to TRPDRV_STAGE_THREADS host threads, default up to 16; the i-role and k-role blocks
 * sent to the device only when changed; slices inside registered arrays gathered on the device) and
 * one launch of the fused FP64 kernel computes the energies without writing f; otherwise (or with
 * TRPDRV_DROPIN_PATH=plain) the plain per-triple path runs (16 GEMMs into f, then the tengy
 * reduction).  The call returns after the energies are back on the host.
 * Errors (bad sizes/indices, CUDA failure) print to stderr and abort, unless TRPDRV_ON_ERROR=return,
 * in which case emp4/emp5 are left unchanged and trpdrv_last_error() reports the status. */
void ccsd_trpdrv_omp_cbody_(double *f1n, double *f1t, double *f2n, double *f2t,
                            double *f3n, double *f3t, double *f4n, double *f4t, double *eorb,
                            int *ncor, int *nocc, int *nvir, double *emp4, double *emp5,
                            int *a, int *i, int *j, int *k, int *klo,
                            double *tij, double *tkj, double *tia, double *tka,
                            double *xia, double *xka, double *jia, double *jka,
                            double *kia, double *kka, double *jij, double *jkj,
                            double *kij, double *kkj,
                            double *dintc1, double *dintx1, double *t1v1,
                            double *dintc2, double *dintx2, double *t1v2);

/* Same contract; replaces the Fortran-77 body ccsd_trpdrv_omp_fbody (omp/ccsd_trpdrv_omp_f77.f:1-9),
 * which omp/test.c calls under -DUSE_FORTRAN (omp/test.c:24-37, 167-171). */
void ccsd_trpdrv_omp_fbody_(double *f1n, double *f1t, double *f2n, double *f2t,
                            double *f3n, double *f3t, double *f4n, double *f4t, double *eorb,
                            int *ncor, int *nocc, int *nvir, double *emp4, double *emp5,
                            int *a, int *i, int *j, int *k, int *klo,
                            double *tij, double *tkj, double *tia, double *tka,
                            double *xia, double *xka, double *jia, double *jka,
                            double *kia, double *kka, double *jij, double *jkj,
                            double *kij, double *kkj,
                            double *dintc1, double *dintx1, double *t1v1,
                            double *dintc2, double *dintx2, double *t1v2);

/* Same contract; replaces ccsd_trpdrv_cbody_ (ocl/ccsd_trpdrv_cbody.c:31; ocl/test.c:49-62). */
void ccsd_trpdrv_cbody_(double *f1n, double *f1t, double *f2n, double *f2t,
                        double *f3n, double *f3t, double *f4n, double *f4t, double *eorb,
                        int *ncor, int *nocc, int *nvir, double *emp4, double *emp5,
                        int *a, int *i, int *j, int *k, int *klo,
                        double *tij, double *tkj, double *tia, double *tka,
                        double *xia, double *xka, double *jia, double *jka,
                        double *kia, double *kka, double *jij, double *jkj,
                        double *kij, double *kkj,
                        double *dintc1, double *dintx1, double *t1v1,
                        double *dintc2, double *dintx2, double *t1v2);

/* Same contract; replaces ccsd_trpdrv_opencl_ (ocl/ccsd_trpdrv_opencl.c:31; ocl/test.c:34-47).
 * Unlike that reference body (whose tengy call is commented out, ocl/ccsd_trpdrv_opencl.c:128-131),
 * this one computes the energies. */
void ccsd_trpdrv_opencl_(double *f1n, double *f1t, double *f2n, double *f2t,
                         double *f3n, double *f3t, double *f4n, double *f4t, double *eorb,
                         int *ncor, int *nocc, int *nvir, double *emp4, double *emp5,
                         int *a, int *i, int *j, int *k, int *klo,
                         double *tij, double *tkj, double *tia, double *tka,
                         double *xia, double *xka, double *jia, double *jka,
                         double *kia, double *kka, double *jij, double *jkj,
                         double *kij, double *kkj,
                         double *dintc1, double *dintx1, double *t1v1,
                         double *dintc2, double *dintx2, double *t1v2);

/* The (b,c) energy reduction alone, on caller-provided host f arrays.  The four outputs are
 * OVERWRITTEN (not accumulated).  Replaces ccsd_tengy_omp (omp/ccsd_tengy_c99.c:5-14): scalars
 * by value, C argument order dintc1, dintx1, t1v1, dintc2, dintx2, t1v2. */
void ccsd_tengy_omp(const double *f1n, const double *f1t, const double *f2n, const double *f2t,
                    const double *f3n, const double *f3t, const double *f4n, const double *f4t,
                    const double *dintc1, const double *dintx1, const double *t1v1,
                    const double *dintc2, const double *dintx2, const double *t1v2,
                    const double *eorb, const double eaijk,
                    double *emp4i, double *emp5i, double *emp4k, double *emp5k,
                    const int ncor, const int nocc, const int nvir);

/* Same contract; replaces ccsd_tengy (ocl/ccsd_tengy.c:3-12). */
void ccsd_tengy(const double *f1n, const double *f1t, const double *f2n, const double *f2t,
                const double *f3n, const double *f3t, const double *f4n, const double *f4t,
                const double *dintc1, const double *dintx1, const double *t1v1,
                const double *dintc2, const double *dintx2, const double *t1v2,
                const double *eorb, const double eaijk,
                double *emp4i, double *emp5i, double *emp4k, double *emp5k,
                const int ncor, const int nocc, const int nvir);

/* Fortran binding of the same reduction; replaces the Fortran-77 ccsd_tengy_omp
 * (omp/ccsd_tengy_f77.f:1-5): everything by reference, argument order
 * dintc1, dintc2, dintx1, dintx2, t1v1, t1v2 (differs from the C order above). */
void ccsd_tengy_omp_(const double *f1n, const double *f1t, const double *f2n, const double *f2t,
                     const double *f3n, const double *f3t, const double *f4n, const double *f4t,
                     const double *dintc1, const double *dintc2,
                     const double *dintx1, const double *dintx2,
                     const double *t1v1, const double *t1v2,
                     const double *eorb, const double *eaijk,
                     double *emp4i, double *emp5i, double *emp4k, double *emp5k,
                     const int *ncor, const int *nocc, const int *nvir);

/* ======================================================================================
 * Part 2. Library interface (no reference counterpart unless stated)
 * ====================================================================================== */

/* Status codes. */
enum {
    TRPDRV_OK = 0,
    TRPDRV_ERR_ARG = 1,          /* invalid argument (sizes, indices, NULL pointers) */
    TRPDRV_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    TRPDRV_ERR_NOMEM = 3,        /* device or host allocation failed */
    TRPDRV_ERR_NODEV = 4,        /* no usable sm_100 device */
    TRPDRV_ERR_STATE = 5,        /* call out of order (e.g. execute before data is bound) */
    TRPDRV_ERR_UNSUPPORTED = 6,  /* mode/shape not supported by the selected kernel */
    TRPDRV_ERR_DEVICE = 7        /* a kernel reported an error through its status word */
};

int trpdrv_last_error(void);               /* status of the most recent failing call, this thread */
const char *trpdrv_last_error_message(void);
const char *trpdrv_status_string(int status);
void trpdrv_clear_error(void);
int trpdrv_version(void);                  /* major*10000 + minor*100 + patch */

/* Execution modes. */
enum {
    TRPDRV_MODE_PLAIN = 0,  /* per triple: one grouped launch of the 16 FP64 GEMMs (f to HBM) + tengy */
    TRPDRV_MODE_FUSED = 1,  /* persistent kernel over (triple, tile-pair) work items; f stays on chip */
    TRPDRV_MODE_EMULATED = 2 /* emulated FP64: Ozaki int8 digit slices on the tensor cores (tcgen05),
                                exact int32 sums, FP64 recombination; FP64 energies (see `slices`) */
};

/* One system: all (i,j,k) triples of one fixed virtual `a`, every reference pointer a slice:
 *   t2    [nocc j][nocc x][nvir][nvir]   tij = t2[j][i],  tkj = t2[j][k]
 *   jvv   [nocc x][nvir][nvir]           jia = jvv[i],    jka = jvv[k]     (kvv likewise)
 *   tov   [nocc x][nvir*nocc]            tia = tov[i],    tka = tov[k]     (xov likewise)
 *   jov   [nocc j][nocc x][nocc*nvir]    jij = jov[j][i], jkj = jov[j][k]  (kov likewise)
 *   dintc, dintx, t1v [nocc x][nvir]     dintc1 = dintc[i], dintc2 = dintc[k], ...
 *   eorb  [ncor+nocc+nvir]
 * `a` is the 1-based orbital index used for eaijk = eorb[a] - (eorb[ncor+i]+eorb[ncor+j]+eorb[ncor+k])
 * (omp/ccsd_trpdrv_omp_cbody.c:126).  Pointers are host or device memory depending on the call. */
typedef struct trpdrv_system {
    int ncor, nocc, nvir, a;
    const double *eorb;
    const double *t2;
    const double *jvv, *kvv;
    const double *tov, *xov;
    const double *jov, *kov;
    const double *dintc, *dintx, *t1v;
} trpdrv_system;

typedef struct trpdrv_options {
    int mode;         /* TRPDRV_MODE_*; default FUSED */
    int nkpass;       /* triple order of the reference driver's k-chunking (omp/test.c:97); default 1 */
    int rank, world;  /* process this rank's cost-balanced share of every system; default 0, 1 */
    int device;       /* CUDA device ordinal; default -1 = current */
    int tile;         /* fused tile width (32 is the only compiled width); 0 = default */
    int ctas_per_sm;  /* fused persistent grid = ctas_per_sm * SM count; 0 = default */
    int use_graph;    /* capture trpdrv_plan_execute's launch sequence in a CUDA graph; default 1 */
    int mma_k;        /* FP64 MMA shape of the fused kernel: 8 = m16n8k8 (default); 16 = m16n8k16 (TMA
                         staging only; cp.async staging then uses 8); 4 = m16n8k4 (cp.async staging only;
                         TMA staging then uses 8) */
    int staging;      /* fused-kernel operand staging: 0 = TMA where supported (even nvir and nocc,
                         16-byte aligned tensors, <= 8 systems), else cp.async; 1 = cp.async; 2 = TMA
                         or fail with TRPDRV_ERR_UNSUPPORTED */
    int slices;       /* EMULATED: base-128 digits per operand element, 4..8; 0 = default (7) */
    int batch;        /* EMULATED: triples per contraction launch (their f fill one half of a double
                         buffer that the energy stage reads back); 0 = default (64) */
    int a_count;      /* full (T) sweep: every system covers the virtual indices a .. a + a_count - 1 (1-based,
                         all within the basis).  The a-dependent tensors (trpdrv_tensor_a_dependent: jvv,
                         kvv, dintc, dintx, t1v) then hold a_count consecutive blocks, a-major; the others
                         are shared.  Energies sum over every (a, i, j, k); per-triple records are
                         [a][triple].  0 or 1 = the single `a` of the reference driver (default). */
    int target_digits;  /* EMULATED: when > 0, digit slices are chosen for a relative error of 10^-target_digits:
                           the plan holds 8 slices, runs 8 until trpdrv_plan_autotune has measured on a
                           sample which fewest slices agree with 8 to 10^-(target_digits+1) */
    int reserved[2];
} trpdrv_options;

void trpdrv_options_default(trpdrv_options *opt);

typedef struct trpdrv_plan trpdrv_plan;

/* Allocates device storage and work queues for nsys systems (only ncor/nocc/nvir/a of `shape` are
 * read).  Returns TRPDRV_OK and sets *plan. */
int trpdrv_plan_create(trpdrv_plan **plan, const trpdrv_system *shape, int nsys,
                       const trpdrv_options *opt);
/* Copies every host tensor of `host` (nsys entries, same shapes) into the plan's device storage
 * (host->device inside this call; pinned host memory makes it faster).  stream may be NULL. */
int trpdrv_plan_upload(trpdrv_plan *plan, const trpdrv_system *host, void *stream);
/* trpdrv_plan_upload followed by trpdrv_plan_execute, with the copies overlapped with the kernels
 * (fused form).  The tensors every j reads (eorb, J, K, TOV, XOV, dintc, dintx, t1v) are copied
 * first; T2, JOV and KOV, which a triple (i, j, k) reads only at block j, are copied on a second
 * stream in `chunks` spans of the processing order (0 = 16), each span's kernel launch waiting only
 * for its own j blocks.  Energies and records are bit-identical to upload + execute.  Other modes
 * run upload + execute (the emulated form slices all of T2 before its first product).  The host
 * tensors must stay unchanged until trpdrv_plan_energies returns; pinned host memory makes the
 * copies asynchronous.  No counterpart in the reference (its driver has no device copies). */
int trpdrv_plan_upload_execute(trpdrv_plan *plan, const trpdrv_system *host, int chunks, void *stream);
/* Uses caller-owned DEVICE tensors instead (no copy).  They must stay valid until the next
 * upload/bind or destroy. */
int trpdrv_plan_bind_device(trpdrv_plan *plan, const trpdrv_system *dev);
/* Enqueues the whole job on `stream` (NULL = the plan's stream).  Asynchronous. */
int trpdrv_plan_execute(trpdrv_plan *plan, void *stream);
/* Waits for the job and returns this rank's per-system totals emp4[s], emp5[s] (compensated sums
 * of emp4i + [i!=k] emp4k over the rank's triples).  Either output may be NULL. */
int trpdrv_plan_energies(trpdrv_plan *plan, double *emp4, double *emp5);
/* This rank's records of system `sys`: n_a * (its triples), a-major; trpdrv_plan_triples writes the
 * triple of record t, ijk[3*t..] = i, j, k (1-based), in the driver order of this rank's share (the
 * same for every a). */
int64_t trpdrv_plan_num_triples(const trpdrv_plan *plan, int sys);
int trpdrv_plan_triples(const trpdrv_plan *plan, int sys, int32_t *ijk);
/* Per-triple records of system `sys` after a job: rec[4*t..] = emp4i, emp5i, emp4k, emp5k. */
int trpdrv_plan_triple_energies(trpdrv_plan *plan, int sys, double *rec);
/* Operand staging the plan's fused kernel uses: 1 = cp.async, 2 = TMA (0 for plain plans or
 * before data is bound). */
int trpdrv_plan_staging(const trpdrv_plan *plan);
/* Kernel launches the last execute enqueued (for launch accounting). */
int64_t trpdrv_plan_last_launches(const trpdrv_plan *plan);
/* Device-time (ms) of the last execute's main kernel(s), measured with events on the plan stream. */
int trpdrv_plan_last_kernel_ms(trpdrv_plan *plan, double *ms);
int trpdrv_plan_destroy(trpdrv_plan *plan);

/* Autotuner: times every compiled variant of the plan's mode on a sample of the plan's own work and
 * keeps the fastest (FUSED: TMA vs cp.async staging, FP64 MMA shape (TMA m16n8k8 / m16n8k16, cp.async
 * m16n8k8 / m16n8k4), edge tile shape (TMA: packed 2 x 32x16 or 32x32 items), CTAs per SM;
 * EMULATED: triples per launch, 8 / 16 / 32 / 64).  Needs a bound plan (after upload or bind); each
 * system is sampled (about 1/8 of its fused items, 64 triples in the emulated form) and the per-
 * system times are scaled to its full work.  EMULATED plans with target_digits first pick the fewest
 * slices (4..8) that meet the accuracy target on the same sample.  The choice is cached per device and set of shapes for
 * the life of the process; a later plan with the same key takes it without timing.  With
 * TRPDRV_TUNE_CACHE naming a file, choices are also appended there (one text line each, keyed by the
 * device model, the library version and the plan's shapes and options) and read back by later
 * processes.  result->from_cache: 0 = timed now, 1 = this process's cache, 2 = the file.  No
 * counterpart in the reference (its BLAS call sites have nothing to tune).  `result` may be NULL. */
typedef struct trpdrv_tune_candidate {
    int staging;          /* FUSED: 1 cp.async, 2 TMA; 0 otherwise */
    int mma_k;            /* FUSED: FP64 MMA shape k (TMA: 8 or 16; cp.async: 4 or 8) */
    int ctas_per_sm;      /* FUSED cp.async grid */
    int batch;            /* EMULATED: triples per contraction launch */
    int edge_pack;        /* FUSED TMA: 1 = where the last tile holds at most 16 virtual indices, its tile
                             pairs run two to a work item (2 x 32x16 tiles); 0 = one 32x32 pair per item */
    double ms_estimate;   /* estimated device time of one execution with this candidate */
} trpdrv_tune_candidate;
typedef struct trpdrv_tune_result {
    int ncand, chosen, from_cache;
    trpdrv_tune_candidate cand[8];
    int slices;           /* EMULATED: digit slices in use after tuning */
    double est_rel_err;   /* EMULATED with target_digits: sampled per-triple deviation of that slice
                             count from 8 slices (normwise per energy column), else 0 */
} trpdrv_tune_result;
int trpdrv_plan_autotune(trpdrv_plan *plan, trpdrv_tune_result *result);

/* One call from host tensors to totals: create, upload, execute, energies, destroy. */
int trpdrv_run(const trpdrv_system *host, int nsys, const trpdrv_options *opt,
               double *emp4, double *emp5);

/* ---- host-side helpers (no device needed) ---- */

/* Number of triples of the reference driver for one `a`: nocc*nocc*(nocc+1)/2 (omp/test.c:160-165). */
int64_t trpdrv_count_triples(int nocc);
/* The driver's triple order for a given nkpass (omp/test.c:97, 160-165): ijkl[4*t..] = i, j, k, klo. */
int64_t trpdrv_enumerate_triples(int nocc, int nkpass, int32_t *ijkl);
/* Splits n items with costs cost[] into `world` contiguous ranges of near-equal total cost:
 * rank r gets [bounds[r], bounds[r+1]). */
int trpdrv_partition(const double *cost, int64_t n, int world, int64_t *bounds);
/* This rank's share of one system's triples, as plans assign them: the driver order for nkpass,
 * split by trpdrv_partition into `world` contiguous ranges of equal count.  Writes ijk[3*t..] =
 * i, j, k (1-based) when ijk is not NULL and returns the share's size (negative on bad arguments). */
int64_t trpdrv_shard_triples(int nocc, int nkpass, int rank, int world, int32_t *ijk);
/* The order in which fused plans process a list of triples (ijk[3*t..] = i, j, k, 1-based, e.g. from
 * trpdrv_shard_triples); energies are still stored and summed in list order, so the order changes
 * no result.  Within each run of equal j the (i, k) triangle is walked in blocks of `block` i values
 * (k outer, direction alternating from block to block, i inner), so that the operand slices one
 * stretch of work touches fit in L2.  Writes the permutation order[position] = list index; returns
 * 0, or -1 on bad arguments.  block <= 0 selects the default (8). */
int trpdrv_processing_order(const int32_t *ijk, int64_t n, int block, int32_t *order);
/* The spans of a processing order (order[position] = list index, NULL = list order) that
 * trpdrv_plan_upload_execute launches one by one: positions [bounds[s], bounds[s+1]) for
 * s < the returned count (at most `chunks`; bounds needs chunks + 1 entries, bounds[0] = 0 and the
 * last bound = n).  Span s ends at the first change of j at or after position (s+1)*n/chunks, so
 * that a run of equal j is never split.  Returns -1 on bad arguments.  No counterpart in the
 * reference. */
int64_t trpdrv_upload_spans(const int32_t *ijk, const int32_t *order, int64_t n, int chunks, int64_t *bounds);
/* Cost (FLOPs) of one triple of a system: 16*nvir*nvir*(nvir+nocc). */
double trpdrv_triple_flops(int nocc, int nvir);

/* Seeded synthetic inputs (counter-based, identical on every machine).  `tensor` selects which
 * array of trpdrv_system to fill (TRPDRV_T_*); n must equal trpdrv_tensor_elems(tensor, ...).
 * dist TRPDRV_DIST_UNIFORM: T2 in [-0.05,0.05]; tov, xov, t1v in [-0.02,0.02]; integrals
 * (jvv, kvv, jov, kov, dintc, dintx) in [-0.1,0.1]; eorb: core sorted in [-20,-5], occupied sorted
 * in [-2,-0.5], virtual sorted in [0.2,3].  TRPDRV_DIST_LOGUNIFORM: integrals instead have a
 * log-uniform magnitude in [1e-6,1] with a random sign. */
enum { TRPDRV_T_EORB = 0, TRPDRV_T_T2, TRPDRV_T_JVV, TRPDRV_T_KVV, TRPDRV_T_TOV, TRPDRV_T_XOV,
       TRPDRV_T_JOV, TRPDRV_T_KOV, TRPDRV_T_DINTC, TRPDRV_T_DINTX, TRPDRV_T_T1V, TRPDRV_T_COUNT };
enum { TRPDRV_DIST_UNIFORM = 0, TRPDRV_DIST_LOGUNIFORM = 1 };
size_t trpdrv_tensor_elems(int tensor, int ncor, int nocc, int nvir);
/* 1 if the tensor carries the virtual index a in a sweep (options.a_count > 1: a_count blocks of
 * trpdrv_tensor_elems each), else 0.  No counterpart in the reference (its driver fixes a). */
int trpdrv_tensor_a_dependent(int tensor);
int trpdrv_synth_fill(int tensor, int ncor, int nocc, int nvir, uint64_t seed, int dist,
                      double *out, size_t n);

/* ---- one triple without device allocation ----
 * No counterpart in the reference.  For callers that cannot call cudaMalloc when they need the work
 * done: a host application that reserves device memory up front in its own pool and gives libraries
 * a fixed budget, a plug-in inside a framework that owns every device buffer, or a loop that cannot
 * pay for an allocation (which may synchronise the device) on every call.
 * Runs the body of one triple (a,i,j,k) on DEVICE pointers that are already sliced for the triple
 * (tkj is the (k,j) block itself, not the k-chunk base; likewise jka, kka, tka, xka, jkj, kkj;
 * dintc2/dintx2/t1v2 are the k vectors) and writes out4[0..3] = emp4i, emp5i, emp4k, emp5k on the
 * device.  Enqueues on `stream` and returns without waiting; allocates nothing: its scratch is one
 * static device array of about 4.7 MB per GPU, kept until the process exits, that limits the size
 * to nvir <= TRPDRV_NOALLOC_MAX_NVIR and nocc <= TRPDRV_NOALLOC_MAX_NOCC (larger sizes are
 * rejected with TRPDRV_ERR_ARG).  All calls on a device share that array: calls that overlap on
 * the GPU race and must be serialised by the caller.  The first call on each device looks up the
 * array and sets kernel attributes; make it before any stream capture.  `a` may be any orbital
 * 1..ncor+nocc+nvir, as in the reference body, whose own driver passes a = 1 (omp/test.c:162); a
 * virtual a (> ncor+nocc) is the physical case.  A CUDA error already pending on the calling thread
 * makes the call return TRPDRV_ERR_STATE without enqueuing anything (the error is left in place). */
#define TRPDRV_NOALLOC_MAX_NVIR 256
#define TRPDRV_NOALLOC_MAX_NOCC 64
typedef struct trpdrv_body_device_args {
    int ncor, nocc, nvir;
    int a, i, j, k;  /* 1-based, as in the reference body.  a is accepted over 1 .. ncor + nocc + nvir
                        like the reference body's (the reference driver itself passes a = 1,
                        omp/test.c:162); a physical sweep passes virtual indices,
                        ncor + nocc < a <= ncor + nocc + nvir, which keep every denominator negative */
    const double *eorb;
    const double *tij, *tkj, *tia, *tka, *xia, *xka, *jia, *jka, *kia, *kka;
    const double *jij, *jkj, *kij, *kkj;
    const double *dintc1, *dintx1, *t1v1, *dintc2, *dintx2, *t1v2;
    double *out4;
} trpdrv_body_device_args;
int trpdrv_body_device_noalloc(const trpdrv_body_device_args *args, void *stream);

/* ---- inputs that do not change between drop-in calls ----
 * The drop-in entry points copy every input slice host -> device on each call, because the
 * reference's callers may refill their buffers between calls (the NWChem driver refills the same
 * host buffers per (i, a) and (k, j) block).  A caller whose arrays stay fixed while
 * it loops over triples (omp/test.c:160-195 passes slices of arrays allocated once) registers them:
 * the library keeps a device copy of [ptr, ptr + bytes), and every drop-in pointer that lies inside
 * a registered array is read from that copy, with no per-call transfer.  After changing a registered
 * array, call trpdrv_refresh_host (or unregister it).  Ranges must not overlap; at most 64 arrays.
 * trpdrv_finalize drops every registration.  No counterpart in the reference (its body reads host
 * memory directly). */
int trpdrv_register_host(const void *ptr, size_t bytes);
int trpdrv_refresh_host(const void *ptr);
int trpdrv_unregister_host(const void *ptr);

/* Releases the drop-in entry points' device state (buffers, stream, registered arrays).  Safe to
 * call repeatedly. */
void trpdrv_finalize(void);

/* Failure-detection self-test.  Every mbarrier wait inside the TMA FP64 kernel and the int8
 * emulated kernel (stage fills, stage releases, accumulator handoffs) gives up after a time limit
 * (4 s), sets an error bit in the launch's status word and returns, so a stalled pipeline ends as
 * TRPDRV_ERR_DEVICE instead of a hung device.  This call runs
 * that same bounded wait on an mbarrier that nothing completes, with the given limit (seconds, in
 * (0, 10]), on the current device: *status receives the kernel's status word (2 = the wait gave
 * up, as it must; 4 = it reported a phase that never completed) and *elapsed_seconds how long the
 * wait lasted.  The device stays usable afterwards.  No counterpart in the reference. */
int trpdrv_selftest_bounded_wait(double limit_seconds, int *status, double *elapsed_seconds);

#ifdef __cplusplus
}
#endif
#endif /* TRPDRV_B200_H */
