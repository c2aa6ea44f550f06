// C ABI: the reference's eleven entry points (src/pt.h), their device-pointer
// twins, and the plan API.  See include/pt.h for the contract of each.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include "plan.h"
#include "pt.h"

#define LIBPT_API extern "C" __attribute__((visibility("default")))

namespace {

void *(*g_malloc)(size_t) = malloc;
void (*g_free)(void *) = free;

// Precision of the FP32 (*_mp) entry points: the FP32 tensor-core form (5
// INT8 digit planes, exact accumulation), or under LIBPT_MP_PRECISION the
// FP64 engine (=fp64) or the 3xTF32 form (=tf32x3; its truncating FP32
// accumulation leaves ~2e-6 relative error in synthetic energies).
int mp_precision() {
  const char *e = getenv("LIBPT_MP_PRECISION");
  if (e && (e[0] == 't' || e[0] == 'T')) return LIBPT_PREC_TF32X3;
  if (e && (e[0] == 'f' || e[0] == 'F') && e[1] == 'p' && e[2] == '6')
    return LIBPT_PREC_FP64;
  return LIBPT_PREC_FP32;
}

// Precision of the FP64 entry points: the FP64 engine, or emulated FP64
// when LIBPT_FP64_PRECISION=emu64 (digit slices chosen per solve for the
// LIBPT_EMU_TOL tolerance, default 1e-6 Eh) or emu64:S (S = 4..7 fixed).
int fp64_precision() {
  const char *e = getenv("LIBPT_FP64_PRECISION");
  if (!e || (e[0] != 'e' && e[0] != 'E')) return LIBPT_PREC_FP64;
  const char *c = e;
  while (*c && *c != ':') ++c;
  const int s = *c ? atoi(c + 1) : 0;
  return LIBPT_PREC_EMU64 | ((s >= 4 && s <= 7 ? s : 0) << 8);
}

[[noreturn]] void fatal(const char *where) {
  fprintf(stderr, "libpt: %s: %s\n", where, ptb::last_error());
  abort();
}

// Host-pointer solve: stage the caller's arrays to the current device, run
// every triple, return the energy.  Aborts on failure like the reference
// (src/pt.c:208-209).
double host_solve(const char *name, int kind, size_t oa, size_t va, size_t ob,
                  size_t vb, const void *const *args, int dtype) {
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    ptb::set_error(cudaGetErrorString(cudaGetLastError()));
    fatal(name);
  }
  libpt_plan *p = nullptr;
  double e = 0.0;
  const double t0 = ptb::wall_seconds();
  // OVVV copies streamed by occupied index next to the triples that need them
  int r = ptb::plan_create(kind, oa, va, ob, vb, args, dtype,
                           dtype ? mp_precision() : fp64_precision(), true, st,
                           &p, nullptr, 0, 0, true);
  const double t1 = ptb::wall_seconds();
  if (!r) r = ptb::plan_run_streamed(p);
  if (!r) r = ptb::plan_energy(p, nullptr, 0, &e);
  if (!r && ptb::profile_enabled())
    fprintf(stderr,
            "libpt: %s oa=%zu va=%zu ob=%zu vb=%zu: upload %.3f s, prepare "
            "%.3f s, tune %.3f s, create %.3f s, triples %.3f s, "
            "precision %d, slices %d\n",
            name, oa, va, ob, vb, p->prof_upload, p->prof_prepare,
            p->prof_tune, t1 - t0, ptb::wall_seconds() - t1, p->precision,
            p->precision == LIBPT_PREC_EMU64 ? p->slices : 0);
  ptb::plan_destroy(p);
  cudaStreamDestroy(st);
  if (r) fatal(name);
  return e;
}

int dev_solve(int kind, size_t oa, size_t va, size_t ob, size_t vb,
              const void *const *args, int dtype, void *stream,
              double *e_out) {
  if (!e_out) {
    ptb::set_error("e_out is NULL");
    return LIBPT_ERR_ARG;
  }
  libpt_plan *p = nullptr;
  int r = ptb::plan_create(kind, oa, va, ob, vb, args, dtype,
                           dtype ? mp_precision() : fp64_precision(), false,
                           static_cast<cudaStream_t>(stream), &p);
  if (!r) r = ptb::plan_run(p, nullptr, p->queue.size());
  if (!r) r = ptb::plan_energy(p, nullptr, 0, e_out);
  ptb::plan_destroy(p);
  return r;
}

}  // namespace

// ---- reference API ----------------------------------------------------------

LIBPT_API void libpt_print_banner(void) {
  printf("libpt-b200: perturbative triples corrections on NVIDIA B200\n");
  printf("drop-in for the libpt C API (CCSD(T), EOM-CCSD(fT))\n");
  printf("https://github.com/ilyak/libpt\n");
}

LIBPT_API void libpt_set_malloc(void *(*fn)(size_t)) {
  g_malloc = fn ? fn : malloc;
}

LIBPT_API void libpt_set_free(void (*fn)(void *)) { g_free = fn ? fn : free; }

LIBPT_API double libpt_rpt(size_t oa, size_t va, const double *d_ov,
                           const double *f_ov, const double *t1,
                           const double *t2, const double *i_oovo,
                           const double *i_oovv, const double *i_ovvv) {
  const void *a[] = {d_ov, f_ov, t1, t2, i_oovo, i_oovv, i_ovvv};
  return host_solve("libpt_rpt", 0, oa, va, oa, va, a, 0);
}

LIBPT_API double libpt_rpt_mp(size_t oa, size_t va, const float *d_ov,
                              const float *f_ov, const float *t1,
                              const float *t2, const float *i_oovo,
                              const float *i_oovv, const float *i_ovvv) {
  const void *a[] = {d_ov, f_ov, t1, t2, i_oovo, i_oovv, i_ovvv};
  return host_solve("libpt_rpt_mp", 0, oa, va, oa, va, a, 1);
}

LIBPT_API double libpt_upt(size_t oa, size_t va, size_t ob, size_t vb,
                           const double *d_ov, const double *f_ov,
                           const double *t1, const double *t2,
                           const double *i_oovo, const double *i_oovv,
                           const double *i_ovvv) {
  const void *a[] = {d_ov, f_ov, t1, t2, i_oovo, i_oovv, i_ovvv};
  return host_solve("libpt_upt", 1, oa, va, ob, vb, a, 0);
}

LIBPT_API double libpt_upt_mp(size_t oa, size_t va, size_t ob, size_t vb,
                              const float *d_ov, const float *f_ov,
                              const float *t1, const float *t2,
                              const float *i_oovo, const float *i_oovv,
                              const float *i_ovvv) {
  const void *a[] = {d_ov, f_ov, t1, t2, i_oovo, i_oovv, i_ovvv};
  return host_solve("libpt_upt_mp", 1, oa, va, ob, vb, a, 1);
}

LIBPT_API double libpt_rft(size_t oa, size_t va, const double *d_ov,
                           const double *f2_ov, const double *l1,
                           const double *t2, const double *l2,
                           const double *i_oovv, const double *i2_t2f2_oovo,
                           const double *i3_ovvv, const double *i6_oovo,
                           const double *i7_ovvv) {
  const void *a[] = {d_ov,   f2_ov,        l1,      t2,      l2,
                     i_oovv, i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv};
  return host_solve("libpt_rft", 2, oa, va, oa, va, a, 0);
}

LIBPT_API double libpt_rft_mp(size_t oa, size_t va, const float *d_ov,
                              const float *f2_ov, const float *l1,
                              const float *t2, const float *l2,
                              const float *i_oovv, const float *i2_t2f2_oovo,
                              const float *i3_ovvv, const float *i6_oovo,
                              const float *i7_ovvv) {
  const void *a[] = {d_ov,   f2_ov,        l1,      t2,      l2,
                     i_oovv, i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv};
  return host_solve("libpt_rft_mp", 2, oa, va, oa, va, a, 1);
}

LIBPT_API double libpt_uft(size_t oa, size_t va, size_t ob, size_t vb,
                           const double *d_ov, const double *f2_ov,
                           const double *l1, const double *t2,
                           const double *l2, const double *i_oovv,
                           const double *i2_t2f2_oovo, const double *i3_ovvv,
                           const double *i6_oovo, const double *i7_ovvv) {
  const void *a[] = {d_ov,   f2_ov,        l1,      t2,      l2,
                     i_oovv, i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv};
  return host_solve("libpt_uft", 3, oa, va, ob, vb, a, 0);
}

LIBPT_API double libpt_uft_mp(size_t oa, size_t va, size_t ob, size_t vb,
                              const float *d_ov, const float *f2_ov,
                              const float *l1, const float *t2,
                              const float *l2, const float *i_oovv,
                              const float *i2_t2f2_oovo, const float *i3_ovvv,
                              const float *i6_oovo, const float *i7_ovvv) {
  const void *a[] = {d_ov,   f2_ov,        l1,      t2,      l2,
                     i_oovv, i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv};
  return host_solve("libpt_uft_mp", 3, oa, va, ob, vb, a, 1);
}

LIBPT_API const char *libpt_last_error(void) { return ptb::last_error(); }

// ---- device-pointer twins ---------------------------------------------------

LIBPT_API int libpt_rpt_dev(size_t oa, size_t va, const double *d_ov,
                            const double *f_ov, const double *t1,
                            const double *t2, const double *i_oovo,
                            const double *i_oovv, const double *i_ovvv,
                            void *stream, double *e_out) {
  const void *a[] = {d_ov, f_ov, t1, t2, i_oovo, i_oovv, i_ovvv};
  return dev_solve(0, oa, va, oa, va, a, 0, stream, e_out);
}

LIBPT_API int libpt_upt_dev(size_t oa, size_t va, size_t ob, size_t vb,
                            const double *d_ov, const double *f_ov,
                            const double *t1, const double *t2,
                            const double *i_oovo, const double *i_oovv,
                            const double *i_ovvv, void *stream,
                            double *e_out) {
  const void *a[] = {d_ov, f_ov, t1, t2, i_oovo, i_oovv, i_ovvv};
  return dev_solve(1, oa, va, ob, vb, a, 0, stream, e_out);
}

LIBPT_API int libpt_rft_dev(size_t oa, size_t va, const double *d_ov,
                            const double *f2_ov, const double *l1,
                            const double *t2, const double *l2,
                            const double *i_oovv, const double *i2_t2f2_oovo,
                            const double *i3_ovvv, const double *i6_oovo,
                            const double *i7_ovvv, void *stream,
                            double *e_out) {
  const void *a[] = {d_ov,   f2_ov,        l1,      t2,      l2,
                     i_oovv, i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv};
  return dev_solve(2, oa, va, oa, va, a, 0, stream, e_out);
}

LIBPT_API int libpt_uft_dev(size_t oa, size_t va, size_t ob, size_t vb,
                            const double *d_ov, const double *f2_ov,
                            const double *l1, const double *t2,
                            const double *l2, const double *i_oovv,
                            const double *i2_t2f2_oovo, const double *i3_ovvv,
                            const double *i6_oovo, const double *i7_ovvv,
                            void *stream, double *e_out) {
  const void *a[] = {d_ov,   f2_ov,        l1,      t2,      l2,
                     i_oovv, i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv};
  return dev_solve(3, oa, va, ob, vb, a, 0, stream, e_out);
}

LIBPT_API int libpt_rpt_mp_dev(size_t oa, size_t va, const float *d_ov,
                               const float *f_ov, const float *t1,
                               const float *t2, const float *i_oovo,
                               const float *i_oovv, const float *i_ovvv,
                               void *stream, double *e_out) {
  const void *a[] = {d_ov, f_ov, t1, t2, i_oovo, i_oovv, i_ovvv};
  return dev_solve(0, oa, va, oa, va, a, 1, stream, e_out);
}

LIBPT_API int libpt_upt_mp_dev(size_t oa, size_t va, size_t ob, size_t vb,
                               const float *d_ov, const float *f_ov,
                               const float *t1, const float *t2,
                               const float *i_oovo, const float *i_oovv,
                               const float *i_ovvv, void *stream,
                               double *e_out) {
  const void *a[] = {d_ov, f_ov, t1, t2, i_oovo, i_oovv, i_ovvv};
  return dev_solve(1, oa, va, ob, vb, a, 1, stream, e_out);
}

LIBPT_API int libpt_rft_mp_dev(size_t oa, size_t va, const float *d_ov,
                               const float *f2_ov, const float *l1,
                               const float *t2, const float *l2,
                               const float *i_oovv,
                               const float *i2_t2f2_oovo,
                               const float *i3_ovvv, const float *i6_oovo,
                               const float *i7_ovvv, void *stream,
                               double *e_out) {
  const void *a[] = {d_ov,   f2_ov,        l1,      t2,      l2,
                     i_oovv, i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv};
  return dev_solve(2, oa, va, oa, va, a, 1, stream, e_out);
}

LIBPT_API int libpt_uft_mp_dev(size_t oa, size_t va, size_t ob, size_t vb,
                               const float *d_ov, const float *f2_ov,
                               const float *l1, const float *t2,
                               const float *l2, const float *i_oovv,
                               const float *i2_t2f2_oovo,
                               const float *i3_ovvv, const float *i6_oovo,
                               const float *i7_ovvv, void *stream,
                               double *e_out) {
  const void *a[] = {d_ov,   f2_ov,        l1,      t2,      l2,
                     i_oovv, i2_t2f2_oovo, i3_ovvv, i6_oovo, i7_ovvv};
  return dev_solve(3, oa, va, ob, vb, a, 1, stream, e_out);
}

// ---- plans --------------------------------------------------------------------

LIBPT_API int libpt_plan_create(int kind, size_t oa, size_t va, size_t ob,
                                size_t vb, const void *const *args, int dtype,
                                int precision, void *stream,
                                libpt_plan **out) {
  if (!out) {
    ptb::set_error("out is NULL");
    return LIBPT_ERR_ARG;
  }
  return ptb::plan_create(kind, oa, va, ob, vb, args, dtype, precision, false,
                          static_cast<cudaStream_t>(stream), out);
}

LIBPT_API int64_t libpt_plan_queue_length(const libpt_plan *plan) {
  return plan ? (int64_t)plan->queue.size() : -1;
}

LIBPT_API int libpt_plan_slices(const libpt_plan *plan) {
  // (the FP32 form runs as emulated FP64 with 4 slices)
  return plan && plan->precision == LIBPT_PREC_EMU64 ? plan->slices : 0;
}

LIBPT_API double libpt_plan_flops(const libpt_plan *plan, int64_t first,
                                  int64_t n) {
  return plan ? ptb::plan_flops(plan, first, n) : 0.0;
}

LIBPT_API int libpt_plan_run(libpt_plan *plan, const int64_t *idx, size_t n) {
  if (!plan || (!idx && n)) {
    ptb::set_error("libpt_plan_run: NULL argument");
    return LIBPT_ERR_ARG;
  }
  return ptb::plan_run(plan, idx, n);
}

LIBPT_API int libpt_plan_run_all(libpt_plan *plan) {
  if (!plan) {
    ptb::set_error("libpt_plan_run_all: NULL plan");
    return LIBPT_ERR_ARG;
  }
  return ptb::plan_run(plan, nullptr, plan->queue.size());
}

LIBPT_API int libpt_plan_energy(libpt_plan *plan, const int64_t *idx,
                                size_t n, double *e_out) {
  if (!plan || !e_out) {
    ptb::set_error("libpt_plan_energy: NULL argument");
    return LIBPT_ERR_ARG;
  }
  return ptb::plan_energy(plan, idx, n, e_out);
}

// ---- a solve sharded over ranks (src/pt.c:197-221, 474-477) ---------------

LIBPT_API int64_t libpt_shard_entries(int64_t queue_length, int rank, int size,
                                      int64_t *idx) {
  const int64_t n = ptb::shard_entries(queue_length, rank, size, idx);
  if (n < 0) ptb::set_error("libpt_shard_entries: invalid rank or size");
  return n;
}

LIBPT_API int libpt_plan_run_shard(libpt_plan *plan, int rank, int size) {
  if (!plan) {
    ptb::set_error("libpt_plan_run_shard: NULL plan");
    return LIBPT_ERR_ARG;
  }
  return ptb::plan_run_shard(plan, rank, size);
}

LIBPT_API int libpt_plan_energy_slots(libpt_plan *plan, double **slots) {
  if (!plan || !slots) {
    ptb::set_error("libpt_plan_energy_slots: NULL argument");
    return LIBPT_ERR_ARG;
  }
  *slots = plan->e_slot;
  return LIBPT_OK;
}

LIBPT_API int libpt_energy_sum(const double *energies, size_t n,
                               double *e_out) {
  if ((!energies && n) || !e_out) {
    ptb::set_error("libpt_energy_sum: NULL argument");
    return LIBPT_ERR_ARG;
  }
  return ptb::sum_slots(energies, n, nullptr, 0, e_out);
}

LIBPT_API int libpt_plan_timing(libpt_plan *plan, int enable) {
  if (!plan) {
    ptb::set_error("libpt_plan_timing: NULL plan");
    return LIBPT_ERR_ARG;
  }
  plan->timing = enable != 0;
  return LIBPT_OK;
}

LIBPT_API int libpt_plan_kernel_stats(libpt_plan *plan, double *gemm_ms,
                                      int64_t *gemm_launches,
                                      double *gemm_flops, double *epi_ms,
                                      int64_t *launches) {
  if (!plan) {
    ptb::set_error("libpt_plan_kernel_stats: NULL plan");
    return LIBPT_ERR_ARG;
  }
  return ptb::plan_kernel_stats(plan, gemm_ms, gemm_launches, gemm_flops,
                                epi_ms, launches);
}

LIBPT_API int libpt_plan_destroy(libpt_plan *plan) {
  ptb::plan_destroy(plan);
  return LIBPT_OK;
}

// Host allocation hooks (src/misc.c:22-23) for the library's host buffers.
namespace ptb {
void *host_alloc(size_t n) { return g_malloc(n); }
void host_free(void *p) { g_free(p); }
}  // namespace ptb
