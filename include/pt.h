/*
 * libpt-b200: perturbative-triples energy corrections on NVIDIA B200.
 *
 * Drop-in for the reference's C API (ilyak/libpt src/pt.h): the eleven
 * entry points below keep the reference's names, argument order, tensor
 * layouts ("last index fastest", properly (anti-)symmetrised blocks) and
 * return convention.  Arrays are HOST pointers, exactly as in the reference;
 * the library copies them to the current CUDA device, computes there, and
 * returns the energy.  The routines print a message and abort() on a CUDA
 * error (the reference exits on allocation failure, src/pt.c:208-209).
 *
 * The device-pointer twins (libpt_*_dev) take the same tensors already in
 * device memory, run on a caller-supplied stream, never abort, and return a
 * status code (LIBPT_OK ...); the energy is written to *e_out.
 *
 * The plan API (libpt_plan_*) keeps one solve's operands resident on the
 * device so that a caller can run the triples queue in pieces (benchmarks,
 * serving loops) and sum the pieces itself.
 */
#ifndef LIBPT_B200_PT_H
#define LIBPT_B200_PT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference API (src/pt.h:26-178) ------------------------------------ */

/* Replaces src/pt.h:26-27 (src/misc.c:25-31). */
void libpt_print_banner(void);

/* Replaces src/pt.h:29-31 (src/misc.c:33-39).  The hook allocates the
 * library's host-side staging memory; NULL restores malloc. */
void libpt_set_malloc(void *(*fn)(size_t));

/* Replaces src/pt.h:33-35 (src/misc.c:41-47).  NULL restores free. */
void libpt_set_free(void (*fn)(void *));

/* Replaces src/pt.h:64-66 (src/pt.c:454-479): restricted CCSD(T). */
double libpt_rpt(size_t oa, size_t va, const double *d_ov, const double *f_ov,
    const double *t1, const double *t2, const double *i_oovo,
    const double *i_oovv, const double *i_ovvv);

/* Replaces src/pt.h:69-71 (src/ptmp.c:455): FP32 tensors, FP64 result. */
double libpt_rpt_mp(size_t oa, size_t va, const float *d_ov, const float *f_ov,
    const float *t1, const float *t2, const float *i_oovo,
    const float *i_oovv, const float *i_ovvv);

/* Replaces src/pt.h:105-107 (src/pt.c:481-535): unrestricted CCSD(T). */
double libpt_upt(size_t oa, size_t va, size_t ob, size_t vb, const double *d_ov,
    const double *f_ov, const double *t1, const double *t2,
    const double *i_oovo, const double *i_oovv, const double *i_ovvv);

/* Replaces src/pt.h:110-112 (src/ptmp.c:482). */
double libpt_upt_mp(size_t oa, size_t va, size_t ob, size_t vb,
    const float *d_ov, const float *f_ov, const float *t1, const float *t2,
    const float *i_oovo, const float *i_oovv, const float *i_ovvv);

/* Replaces src/pt.h:136-139 (src/pt.c:936-972): restricted EOM-CCSD(fT). */
double libpt_rft(size_t oa, size_t va, const double *d_ov, const double *f2_ov,
    const double *l1, const double *t2, const double *l2, const double *i_oovv,
    const double *i2_t2f2_oovo, const double *i3_ovvv, const double *i6_oovo,
    const double *i7_ovvv);

/* Replaces src/pt.h:142-145 (src/ptmp.c:937). */
double libpt_rft_mp(size_t oa, size_t va, const float *d_ov, const float *f2_ov,
    const float *l1, const float *t2, const float *l2, const float *i_oovv,
    const float *i2_t2f2_oovo, const float *i3_ovvv, const float *i6_oovo,
    const float *i7_ovvv);

/* Replaces src/pt.h:169-172 (src/pt.c:974-1050): unrestricted EOM-CCSD(fT). */
double libpt_uft(size_t oa, size_t va, size_t ob, size_t vb, const double *d_ov,
    const double *f2_ov, const double *l1, const double *t2, const double *l2,
    const double *i_oovv, const double *i2_t2f2_oovo, const double *i3_ovvv,
    const double *i6_oovo, const double *i7_ovvv);

/* Replaces src/pt.h:175-178 (src/ptmp.c:975). */
double libpt_uft_mp(size_t oa, size_t va, size_t ob, size_t vb,
    const float *d_ov, const float *f2_ov, const float *l1, const float *t2,
    const float *l2, const float *i_oovv, const float *i2_t2f2_oovo,
    const float *i3_ovvv, const float *i6_oovo, const float *i7_ovvv);

/* ---- status codes ------------------------------------------------------- */

#define LIBPT_OK             0
#define LIBPT_ERR_ARG        1   /* bad size, NULL pointer, unknown option  */
#define LIBPT_ERR_NOMEM      2   /* device or host allocation failed        */
#define LIBPT_ERR_CUDA       3   /* a CUDA runtime/driver call failed       */
#define LIBPT_ERR_TIMEOUT    4   /* a device-side wait ran out of its limit */
#define LIBPT_ERR_UNSUPPORTED 5  /* option not available on this device     */
#define LIBPT_ERR_CANCELLED  6   /* a served solve was cancelled (pt_serve.h) */

/* Text of the last error on the calling thread ("" if none). */
const char *libpt_last_error(void);

/* ---- precision modes ---------------------------------------------------- */

#define LIBPT_PREC_FP64   0   /* FP64 DMMA tensor-core contractions          */
#define LIBPT_PREC_TF32X3 1   /* 3xTF32 on tcgen05 tensor cores (hi*hi +
                                 hi*lo + lo*hi, FP32 accumulation in TMEM).
                                 The tensor cores' FP32 accumulation
                                 truncates, a bias that adds up coherently
                                 over a solve: ~2e-6 |E| on synthetic
                                 inputs, 1e3-1e4 times the reference *_mp's
                                 own arithmetic error.  Opt-in only
                                 (LIBPT_MP_PRECISION=tf32x3).                 */

#define LIBPT_PREC_EMU64  2   /* emulated FP64: Ozaki-style split of FP64
                                 operands into S signed digit planes (8-bit
                                 balanced digits, or 7-bit ones where the
                                 INT32 bound needs them; power-of-two scale
                                 per row / column), exact INT32 accumulation
                                 of the S(S+1)/2 leading digit products on
                                 tcgen05 INT8 tensor cores.
                                 LIBPT_PREC_EMU64 | (S << 8) fixes S in
                                 [4, 7]; S = 0 lets the plan choose the
                                 smallest S whose error, estimated on a
                                 sample of triples against the most stored
                                 planes, is under LIBPT_EMU_TOL / 2
                                 (environment, Eh; default 1e-6, i.e.
                                 1 uEh).  The FP64 entry points (libpt_rpt
                                 ... and their _dev twins) use it when the
                                 environment sets LIBPT_FP64_PRECISION=emu64
                                 (S chosen) or emu64:S; otherwise they run
                                 FP64 DMMA                                   */

#define LIBPT_PREC_FP32   3   /* the FP32 tensor-core form, default of the
                                 *_mp entry points: FP32 inputs split into 5
                                 INT8 digit planes (39-bit significands,
                                 beyond FP32's 24), digits rounded to
                                 nearest, exact INT32 accumulation on tcgen05
                                 INT8 tensor cores, energy terms in FP64.
                                 Unlike FP32 accumulation (rounded or
                                 truncated), its per-element error is both
                                 unbiased and far below FP32 rounding, so
                                 the result carries the rounding of the FP32
                                 inputs themselves plus an arithmetic error
                                 under 1 % of the reference's sgemm_ path's
                                 (src/ptmp.c:28-38).  LIBPT_MP_PRECISION=fp64
                                 evaluates the FP32 inputs with the FP64
                                 engine instead, =tf32x3 with 3xTF32.  A
                                 plan reports 5 slices.                      */

/* Built-in self-test of a contraction kernel: C = A B1 - A B2 on random
 * m x k and k x n operands, against an FP64 reference computed on the device;
 * writes max|C - C_ref| / max(|A| (|B1| + |B2|)) to *rel_err (the error over
 * the scale that bounds a dot product's rounding).  precision selects the
 * kernel (LIBPT_PREC_*, with the slice count in bits 8-14 for
 * LIBPT_PREC_EMU64, and bit 15 set for 8-bit digit planes -- a signed top
 * digit, unsigned lower digits; S <= 6 -- instead of 7-bit signed digits)
 * and bits 16-23 a tile variant: FP64 0 = 128-row,
 * 1 = 96-row tiles; emulated FP64 the index of one of the slice count's
 * INT8 tile shapes (0 = widest); libpt_selftest_variants() counts them.
 * Bits 24-31 nonzero: the kernel reads its tensor maps from device memory
 * (the form batched multi-solve launches use) instead of kernel parameters.
 * No counterpart in the reference. */
int libpt_selftest(int precision, int m, int n, int k, double *rel_err);
/* Number of tile variants libpt_selftest accepts for a precision (with its
 * slice count in bits 8-15).  No counterpart in the reference. */
int libpt_selftest_variants(int precision);
/* Contraction-kernel microbenchmark: the libpt_selftest job (m x k by
 * k x n, two segments, operands resident in device memory; n up to 2^20
 * with n*k <= 2^27 and m*n <= 2^25) checked once, then launched reps times;
 * writes the mean
 * device time of one launch (ms) and the check's error (rel_err, may be
 * NULL).  The job does 4*m*n*k flops.  No counterpart in the reference. */
int libpt_kernel_bench(int precision, int m, int n, int k, int reps,
                       double *ms, double *rel_err);
/* Failure-detection self-test of the device-side bounded waits: a
 * producer / consumer kernel passes `stages` hand-offs through a ring of
 * mbarriers (as the contraction kernels' pipelines do), but its producer
 * stops after `arrive` of them.  Each wait is limited to limit_ms
 * (0 < limit_ms <= 2000; the kernels' own limit is 2 s): a missing hand-off
 * makes the consumer's wait run out, the kernel records the timeout in its
 * error word and returns, and the call returns LIBPT_ERR_TIMEOUT -- the
 * status a solve reports when one of its kernels' waits runs out; the
 * device stays usable.  *seen = hand-offs the consumer received.  No
 * counterpart in the reference. */
int libpt_selftest_wait(int stages, int arrive, double limit_ms, int *seen);

/* Accuracy of the energy epilogues' reciprocal of the denominators (an
 * approximate reciprocal refined by two Newton-Raphson steps, used in place
 * of a division): *max_ulp = the largest distance, in units in the last
 * place, from the IEEE division 1.0 / d over n values d = +-m * 2^x, x in
 * [lo_exp, hi_exp] (-1000 <= lo_exp <= hi_exp <= 1000), m in [1, 2).  No
 * counterpart in the reference (its energy divides, src/pt.c:291-295). */
int libpt_selftest_recip(int lo_exp, int hi_exp, int n, double *max_ulp);

/* ---- upstream producer (device) -----------------------------------------
 * Builds the restricted (T) inputs of libpt_rpt / libpt_rpt_dev on the
 * device from a density-fitted closed-shell CCSD's results: the
 * three-index factors b_oo[Q][i][j], b_ov[Q][i][a], b_vv[Q][a][b]
 * (naux x o x o, naux x o x v, naux x v x v, row-major, device pointers)
 * give i_oovv abab = (ia|jb), i_ovvv abab = (ib|ac), i_oovo abab = (ia|jk)
 * and their same-spin (aaaa) blocks in the pt.h layout; t2_abab (o x o x v
 * x v, may be t2 + o*o*v*v, or NULL to leave t2 alone) gives t2's aaaa and
 * abab blocks.  Outputs are device arrays of the libpt_rpt sizes.  Work is
 * ordered on `stream` and may still run when the call returns (the GEMMs run
 * through cuBLAS, loaded at the first call; a v^3 scratch block is
 * allocated stream-ordered).  Returns LIBPT_OK or an error code.  No
 * counterpart in the reference (its caller builds these arrays). */
int libpt_rpt_inputs_df(size_t o, size_t v, size_t naux, const double *b_oo,
    const double *b_ov, const double *b_vv, const double *t2_abab,
    double *t2, double *i_oovo, double *i_oovv, double *i_ovvv,
    void *stream);

/* The unrestricted (T) integrals of libpt_upt / libpt_upt_dev from the
 * factors of each spin (b_*_a: alpha, oa x va; b_*_b: beta, ob x vb; same
 * layouts as above): abab blocks (ia|jb), (ib|ac), (ia|jk) with the first
 * occupied and first virtual index alpha, baba the same with the spins
 * exchanged, aaaa / bbbb the antisymmetrised same-spin products.  The
 * amplitudes, spin blocks of their own in an unrestricted CCSD, are not
 * touched.  A factor array with no elements (o or v zero) may be NULL.
 * Same ordering and allocation as libpt_rpt_inputs_df. */
int libpt_upt_inputs_df(size_t oa, size_t va, size_t ob, size_t vb,
    size_t naux, const double *b_oo_a, const double *b_ov_a,
    const double *b_vv_a, const double *b_oo_b, const double *b_ov_b,
    const double *b_vv_b, double *i_oovo, double *i_oovv, double *i_ovvv,
    void *stream);

/* ---- device-pointer twins ----------------------------------------------
 * Same arguments as the reference entry points, but every tensor is a
 * device pointer on the current device and `stream` (a cudaStream_t, may be
 * NULL for the legacy default stream) orders the work.  The call returns
 * when the energy is known.  Scratch memory is allocated with cudaMalloc and
 * released before return.  The *_mp twins take float tensors. */

int libpt_rpt_dev(size_t oa, size_t va, const double *d_ov,
    const double *f_ov, const double *t1, const double *t2,
    const double *i_oovo, const double *i_oovv, const double *i_ovvv,
    void *stream, double *e_out);
int libpt_upt_dev(size_t oa, size_t va, size_t ob, size_t vb,
    const double *d_ov, const double *f_ov, const double *t1, const double *t2,
    const double *i_oovo, const double *i_oovv, const double *i_ovvv,
    void *stream, double *e_out);
int libpt_rft_dev(size_t oa, size_t va, const double *d_ov,
    const double *f2_ov, const double *l1, const double *t2, const double *l2,
    const double *i_oovv, const double *i2_t2f2_oovo, const double *i3_ovvv,
    const double *i6_oovo, const double *i7_ovvv, void *stream,
    double *e_out);
int libpt_uft_dev(size_t oa, size_t va, size_t ob, size_t vb,
    const double *d_ov, const double *f2_ov, const double *l1,
    const double *t2, const double *l2, const double *i_oovv,
    const double *i2_t2f2_oovo, const double *i3_ovvv, const double *i6_oovo,
    const double *i7_ovvv, void *stream, double *e_out);

int libpt_rpt_mp_dev(size_t oa, size_t va, const float *d_ov,
    const float *f_ov, const float *t1, const float *t2, const float *i_oovo,
    const float *i_oovv, const float *i_ovvv, void *stream, double *e_out);
int libpt_upt_mp_dev(size_t oa, size_t va, size_t ob, size_t vb,
    const float *d_ov, const float *f_ov, const float *t1, const float *t2,
    const float *i_oovo, const float *i_oovv, const float *i_ovvv,
    void *stream, double *e_out);
int libpt_rft_mp_dev(size_t oa, size_t va, const float *d_ov,
    const float *f2_ov, const float *l1, const float *t2, const float *l2,
    const float *i_oovv, const float *i2_t2f2_oovo, const float *i3_ovvv,
    const float *i6_oovo, const float *i7_ovvv, void *stream, double *e_out);
int libpt_uft_mp_dev(size_t oa, size_t va, size_t ob, size_t vb,
    const float *d_ov, const float *f2_ov, const float *l1, const float *t2,
    const float *l2, const float *i_oovv, const float *i2_t2f2_oovo,
    const float *i3_ovvv, const float *i6_oovo, const float *i7_ovvv,
    void *stream, double *e_out);

/* ---- allocation-free restricted (T) for small systems ------------------
 * No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory: programs that give all device memory to their own
 * pool allocator up front (a library cudaMalloc would fail or break their
 * accounting) and latency-sensitive loops where cudaMalloc/cudaFree would
 * synchronize the device.  Same arguments and result as libpt_rpt_dev (FP64
 * device tensors in pt.h layout on the current device), but it allocates
 * nothing: all scratch lives in one static device array of
 * LIBPT_STATIC_SCRATCH_BYTES, which every GPU that loads the library's
 * device code keeps until the process exits.  Systems whose scratch does not
 * fit are rejected with LIBPT_ERR_ARG before any work is queued (o = 8,
 * v = 64 fits; the check is the exact footprint of the solve).
 * The first call on a device loads the library's device code there (CUDA
 * loads modules lazily), which reserves the array and the kernels' code, and
 * looks up the array's device address: make that first call -- any size
 * that fits -- before a pool allocator claims the device's memory and before
 * any stream capture.  A call synchronizes the stream it is given (it reads
 * back whether f_ov is zero and the energies), not the device.
 * Every call shares the array: calls whose work overlaps on the GPU race and
 * give wrong results -- serialize them. */
#define LIBPT_STATIC_SCRATCH_BYTES (64ull << 20)

int libpt_rpt_dev_static(size_t oa, size_t va, const double *d_ov,
    const double *f_ov, const double *t1, const double *t2,
    const double *i_oovo, const double *i_oovv, const double *i_ovvv,
    void *stream, double *e_out);

/* ---- plans: resident operands, the triples queue run in pieces ----------
 *
 * A plan holds one solve's operands on the device in the library's padded
 * layout.  Its triples queue lists, in order, the same-spin triples i<j<k of
 * the alpha case, those of the beta case (unrestricted only), the mixed-spin
 * triples i<j (alpha), k (beta), and those of the beta-beta-alpha case
 * (unrestricted only) -- the order of src/pt.c:514-529.  Running every queue
 * entry once and calling libpt_plan_energy gives the solver's result
 * (including the restricted factor 2, src/pt.c:478).
 *
 * kind: 0 = (T) restricted, 1 = (T) unrestricted, 2 = (fT) restricted,
 *       3 = (fT) unrestricted.
 * args: the pt.h tensor pointers of that kind, in the reference's argument
 *       order (7 for (T), 10 for (fT)), DEVICE pointers, FP64 (dtype 0) or
 *       FP32 (dtype 1).  They are read during libpt_plan_create only. */
typedef struct libpt_plan libpt_plan;

int libpt_plan_create(int kind, size_t oa, size_t va, size_t ob, size_t vb,
    const void *const *args, int dtype, int precision, void *stream,
    libpt_plan **out);
/* Number of entries of the triples queue. */
int64_t libpt_plan_queue_length(const libpt_plan *plan);
/* Digit slices an emulated-FP64 plan runs with (its choice when created
 * with S = 0), 0 for the other precision modes. */
int libpt_plan_slices(const libpt_plan *plan);
/* Algorithmic flops of queue entries [first, first+n): twice the
 * multiply-adds of the reference's own contractions for those triples. */
double libpt_plan_flops(const libpt_plan *plan, int64_t first, int64_t n);
/* Compute queue entries idx[0..n) (host array); their energies are stored
 * in the plan (overwriting earlier runs of the same entries).  Asynchronous
 * on the plan's stream. */
int libpt_plan_run(libpt_plan *plan, const int64_t *idx, size_t n);
/* Compute every queue entry (the whole solve).  Asynchronous. */
int libpt_plan_run_all(libpt_plan *plan);
/* Wait for the plan's stream and return the fixed-order, compensated sum of
 * the stored energies of entries idx[0..n) (idx == NULL: all entries), each
 * scaled by the restricted factor 2 (src/pt.c:478) for restricted kinds, so
 * that the sum over the whole queue is the solver's result. */
int libpt_plan_energy(libpt_plan *plan, const int64_t *idx, size_t n,
    double *e_out);
int libpt_plan_destroy(libpt_plan *plan);

/* ---- one solve sharded over ranks (src/pt.c:197-221, 474-477) ----------
 *
 * The reference's MPI scheme on GPUs: every rank (one per GPU) creates a
 * plan from the same inputs and runs the queue entries it owns, entry q
 * belonging to rank q % size (src/pt.c:213, `it % size == rank`).  The
 * ranks then add their per-triple energy slots -- queue_length doubles on
 * the device, zero where another rank owns the entry -- with one in-place
 * sum all-reduce (ncclAllReduce, or MPI_Allreduce on a host copy), the
 * counterpart of the reference's one-double MPI_Allreduce (src/pt.c:
 * 474-477).  libpt_plan_energy on any rank then returns the one-GPU energy
 * bitwise: each slot holds exactly its owner's value, and the sum runs in
 * queue order as for an unsharded solve. */

/* Writes to idx (when non-NULL) the queue entries rank `rank` of `size`
 * owns, in increasing order; returns their number, -1 for invalid
 * arguments.  Host-only: needs no device. */
int64_t libpt_shard_entries(int64_t queue_length, int rank, int size,
    int64_t *idx);
/* Zeroes all of the plan's energy slots, then runs the entries rank `rank`
 * of `size` owns.  Asynchronous on the plan's stream. */
int libpt_plan_run_shard(libpt_plan *plan, int rank, int size);
/* Device address of the plan's per-triple energies (queue_length doubles,
 * queue order, restricted factor not applied).  Valid until the plan is
 * destroyed; the caller may overwrite it (e.g. with an all-reduce) once the
 * plan's stream has finished its runs. */
int libpt_plan_energy_slots(libpt_plan *plan, double **slots);
/* Host-only: the queue-order compensated sum libpt_plan_energy applies
 * (without the restricted factor 2) of energies[0..n). */
int libpt_energy_sum(const double *energies, size_t n, double *e_out);

/* Kernel timing for benchmarks: with timing enabled, each batch records CUDA
 * events around its contraction (GEMM) and energy (epilogue) launches on the
 * plan's stream.  libpt_plan_kernel_stats waits for the stream, returns the
 * summed GEMM time (ms), the number of GEMM launches, their algorithmic flops,
 * the summed epilogue time (ms) and the number of kernels launched by runs
 * since the last call, and resets the counters.  Any pointer may be NULL. */
int libpt_plan_timing(libpt_plan *plan, int enable);
int libpt_plan_kernel_stats(libpt_plan *plan, double *gemm_ms,
    int64_t *gemm_launches, double *gemm_flops, double *epi_ms,
    int64_t *launches);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* LIBPT_B200_PT_H */
