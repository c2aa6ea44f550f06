/*
 * Oracle: a CPU restatement of libpt's perturbative-triples energies.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline arm load this library, and only as the checker.
 * The product (libpt_b200) never calls it.
 *
 * Each function takes the same arguments, in the same order and with the same
 * tensor layouts, as the reference entry point it restates (src/pt.h:64-178):
 *
 *   oracle_rpt  <-> libpt_rpt   (src/pt.c:454-479)
 *   oracle_upt  <-> libpt_upt   (src/pt.c:481-535)
 *   oracle_rft  <-> libpt_rft   (src/pt.c:936-972)
 *   oracle_uft  <-> libpt_uft   (src/pt.c:974-1050)
 *   oracle_*_mp <-> libpt_*_mp  (src/ptmp.c:455, 482, 937, 975): FP32 tensors,
 *                   FP32 contractions and per-element terms, FP64 accumulator.
 *
 * The summation order is fixed (one thread per triple, per-triple partials
 * summed in triple order), so results are reproducible for any thread count.
 */
#ifndef PT_ORACLE_H
#define PT_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

double oracle_rpt(size_t oa, size_t va, const double *d_ov, const double *f_ov,
    const double *t1, const double *t2, const double *i_oovo,
    const double *i_oovv, const double *i_ovvv);
double oracle_upt(size_t oa, size_t va, size_t ob, size_t vb,
    const double *d_ov, const double *f_ov, const double *t1, const double *t2,
    const double *i_oovo, const double *i_oovv, const double *i_ovvv);
double oracle_rft(size_t oa, size_t va, const double *d_ov,
    const double *f2_ov, const double *l1, const double *t2, const double *l2,
    const double *i_oovv, const double *i2_t2f2_oovo, const double *i3_ovvv,
    const double *i6_oovo, const double *i7_ovvv);
double oracle_uft(size_t oa, size_t va, size_t ob, size_t vb,
    const double *d_ov, const double *f2_ov, const double *l1,
    const double *t2, const double *l2, const double *i_oovv,
    const double *i2_t2f2_oovo, const double *i3_ovvv, const double *i6_oovo,
    const double *i7_ovvv);

double oracle_rpt_mp(size_t oa, size_t va, const float *d_ov,
    const float *f_ov, const float *t1, const float *t2, const float *i_oovo,
    const float *i_oovv, const float *i_ovvv);
double oracle_upt_mp(size_t oa, size_t va, size_t ob, size_t vb,
    const float *d_ov, const float *f_ov, const float *t1, const float *t2,
    const float *i_oovo, const float *i_oovv, const float *i_ovvv);
double oracle_rft_mp(size_t oa, size_t va, const float *d_ov,
    const float *f2_ov, const float *l1, const float *t2, const float *l2,
    const float *i_oovv, const float *i2_t2f2_oovo, const float *i3_ovvv,
    const float *i6_oovo, const float *i7_ovvv);
double oracle_uft_mp(size_t oa, size_t va, size_t ob, size_t vb,
    const float *d_ov, const float *f2_ov, const float *l1, const float *t2,
    const float *l2, const float *i_oovv, const float *i2_t2f2_oovo,
    const float *i3_ovvv, const float *i6_oovo, const float *i7_ovvv);

/* Per-triple partial energies of one spin case, in triple order, for
 * debugging the device path: kind 0 = same-spin (aaa) triples i<j<k,
 * kind 1 = mixed-spin (aab) triples i<j, all k.  Restricted (T) inputs.
 * Writes at most `cap` values; returns the number of triples. */
size_t oracle_rpt_partials(int kind, size_t oa, size_t va, const double *d_ov,
    const double *f_ov, const double *t1, const double *t2,
    const double *i_oovo, const double *i_oovv, const double *i_ovvv,
    double *out, size_t cap);

#ifdef __cplusplus
}
#endif

#endif
