// The triples engine, plan creation and life cycle: argument checks, the
// spin-block split of the packed arguments, uploads, operand preparation,
// slice choice and tuning, the sizing pass (footprint) and destruction.
// The other parts are plan_views.cu (tensor maps), plan_upload.cu (device
// memory and uploads), plan_cases.cu (spin cases, job templates, queue),
// plan_emu.cu (emulated FP64 operands), plan_tune.cu (autotuner) and
// plan_run.cu (rounds, energies, sharding).
//
// Reference structure restated here:
//   spin-block split of the packed arguments   src/pt.c:460-467, 487-512,
//                                              943-956, 981-1021
//   spin cases and their block roles           src/pt.c:469-473, 514-529,
//                                              958-966, 1023-1044
//   triple enumeration (i<j<k; i<j, all k)     src/pt.c:210-221, 333-344
//   restricted factor 2                        src/pt.c:478, 971
// The reference's OpenMP/MPI distribution of triples (src/pt.c:197-229)
// becomes batches of triples, each batch one GEMM launch over all of its
// triples' output tiles and one epilogue launch; per-triple energies land in
// slots indexed by queue position and are summed in queue order.
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <mutex>
#include <thread>
#include <vector>

#include "plan_impl.h"
#include "pt.h"

namespace ptb {

static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }

// Sizing pass (plan_footprint): plan creation runs its host logic with
// device allocations carved from a fake arena and every device operation
// skipped, so the arena's high-water mark is the plan's exact footprint.
thread_local bool g_dry = false;

const char *last_error() { return g_last_error.c_str(); }

int plan_create(int kind, size_t oa, size_t va, size_t ob, size_t vb,
                const void *const *args, int dtype, int precision, bool host,
                cudaStream_t st, libpt_plan **out, void *arena,
                size_t arena_size, size_t arena_nb, bool stream_ovvv) {
  *out = nullptr;
  if (kind < 0 || kind > 3 || dtype < 0 || dtype > 1 || !args) {
    set_error("libpt_plan_create: bad kind/dtype/args");
    return LIBPT_ERR_ARG;
  }
  int slices = (precision >> 8) & 0xFF;
  precision &= 0xFF;
  if (precision == LIBPT_PREC_FP32) {
    // the FP32 tensor-core form: the emulated-FP64 engine on 5 digit planes
    // (4 planes leave an arithmetic error up to 0.7 of the reference *_mp's
    // on small systems; 5 keep it below 1 % of it)
    if (slices != 0 && slices != 5) {
      set_error("libpt_plan_create: the FP32 form runs 5 digit slices");
      return LIBPT_ERR_ARG;
    }
    precision = LIBPT_PREC_EMU64;
    slices = 5;
  }
  if (precision != LIBPT_PREC_FP64 && precision != LIBPT_PREC_TF32X3 &&
      precision != LIBPT_PREC_EMU64) {
    set_error("libpt_plan_create: unknown precision mode");
    return LIBPT_ERR_ARG;
  }
  const bool auto_slices = slices == 0;
  if (auto_slices) slices = TC_S_MAX;   // chosen after the planes exist
  if (slices < TC_S_MIN || slices > TC_S_MAX) {
    set_error("libpt_plan_create: emulated FP64 takes 4 to 7 slices");
    return LIBPT_ERR_ARG;
  }
  const bool unr = kind == 1 || kind == 3, ft = kind >= 2;
  if (!unr) {
    ob = oa;
    vb = va;
  }
  const size_t lim = 1u << 15;
  if (oa > lim || va > lim || ob > lim || vb > lim) {
    set_error("libpt_plan_create: orbital space too large");
    return LIBPT_ERR_ARG;
  }
  const int nargs = ft ? 10 : 7;
  for (int a = 0; a < nargs; ++a)
    if (!args[a]) {
      set_error("libpt_plan_create: NULL tensor argument");
      return LIBPT_ERR_ARG;
    }
  const double t_start = wall_seconds();
  libpt_plan *p = new libpt_plan();
  p->kind = kind;
  p->unrestricted = unr;
  p->ft = ft;
  p->oa = (int)oa;
  p->va = (int)va;
  p->ob = (int)ob;
  p->vb = (int)vb;
  p->dtype = dtype;
  p->precision = precision;
  p->slices = slices;
  p->slices_store = slices;
  p->slices_auto = auto_slices && precision == LIBPT_PREC_EMU64;
  p->defer_ovvv = stream_ovvv && host && !unr && oa > 0 && va > 0 &&
                  precision == LIBPT_PREC_FP64;
  if (const char *t = std::getenv("LIBPT_EMU_TOL")) {
    const double v = std::atof(t);
    if (v > 0) p->emu_tol = v;
  }
  {
    const I8Tile *t = nullptr;
    if (i8_tiles(slices, &t) > 0) p->i8tile = t[0];   // widest tile
  }
  p->st = st;
  p->factor = unr ? 1.0 : 2.0;   // src/pt.c:478, 534, 971, 1049
  p->arena = static_cast<char *>(arena);
  p->arena_size = arena ? arena_size : 0;
  int r = LIBPT_OK;
  do {
    Sizes S{(int64_t)oa, (int64_t)va, (int64_t)ob, (int64_t)vb};
    Uploader up{p, host, dtype == 1};
    {
      // staging: no larger than the largest argument array (64 MiB at most)
      int64_t big = (int64_t)(oa * va + (unr ? ob * vb : 0));
      int64_t t2 = 0, oo = 0, vv = 0;
      for (int b = 0; b < (unr ? 4 : 2); ++b) {
        t2 += S.oovv(b);
        oo += S.oovo(b);
        vv += S.ovvv(b);
      }
      big = std::max({big, t2, oo, vv});
      const size_t bytes = (size_t)big * (dtype ? 4 : 8);
      up.stage_cap = std::max<size_t>(256, std::min(up.stage_cap, (bytes + 255) & ~size_t(255)));
      // (two device staging buffers of this size; see Uploader)
    }
    const int64_t nov = (int64_t)(oa * va + (unr ? ob * vb : 0));
    if ((r = dalloc(p, (void **)&p->d_ov, nov * 8 + 8))) break;
    if ((r = dalloc(p, (void **)&p->ov1, nov * 8 + 8))) break;
    if ((r = dalloc(p, (void **)&p->ov2, nov * 8 + 8))) break;
    // (T): d_ov f_ov t1 t2 i_oovo i_oovv i_ovvv
    // (fT): d_ov f2_ov l1 t2 l2 i_oovv i2_t2f2_oovo i3_ovvv i6_oovo i7_ovvv
    const void *a_d = args[0], *a_f = args[1], *a_1 = args[2];
    const void *a_oovv = args[5];
    if ((r = up.put(p->d_ov, a_d, 1, nov, nov))) break;
    if ((r = up.put(p->ov1, a_1, 1, nov, nov))) break;
    if ((r = up.put(p->ov2, a_f, 1, nov, nov))) break;
    const int nb = unr ? 4 : 2;
    const size_t es = dtype ? 4 : 8;
    int64_t off = 0;
    for (int b = 0; b < nb && !r; ++b) {
      const int64_t n = S.oovv(b);
      if ((r = dalloc(p, (void **)&p->oovv[b], n * 8 + 8))) break;
      r = up.put(p->oovv[b], (const char *)a_oovv + off * es, 1, n, n);
      off += n;
    }
    if (r) break;
    if (!unr) p->oovv[3] = p->oovv[1];
    if (!ft) {
      r = upload_set(p, up, S, p->L, args[3], args[4], args[6]);
    } else {
      r = upload_set(p, up, S, p->L, args[4], args[8], args[9]);   // l2, i6, i7
      if (!r) r = upload_set(p, up, S, p->R, args[3], args[6], args[7]);  // t2, i2, i3
    }
    if (r) break;
    p->up_stage[0] = up.stage[0];   // for the deferred OVVV copies
    p->up_stage[1] = up.stage[1];
    p->up_stage_bytes = up.stage_bytes;
    if (!g_dry && cudaStreamSynchronize(st) != cudaSuccess) {
      set_error(std::string("preparing operands: ") +
                cudaGetErrorString(cudaGetLastError()));
      r = LIBPT_ERR_CUDA;
      break;
    }
    p->prof_upload = wall_seconds() - t_start;
    if (!g_dry) {   // an all-zero f_ov (the usual case) skips its terms
      // on the plan's stream (a plain cudaMemcpy would run on the legacy
      // default stream, which waits for every blocking stream of the device)
      std::vector<double> f((size_t)nov);
      if (cudaMemcpyAsync(f.data(), p->ov2, (size_t)nov * 8,
                          cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess) {
        set_error(std::string("reading f_ov: ") +
                  cudaGetErrorString(cudaGetLastError()));
        r = LIBPT_ERR_CUDA;
        break;
      }
      p->has_f = std::any_of(f.begin(), f.end(),
                             [](double x) { return x != 0.0; });
    }
    if ((r = add_cases(p))) break;
    if (p->precision != LIBPT_PREC_FP64) {
      // the tensor-core paths read planes; of the padded FP64 blocks only the
      // amplitudes stay (the energy epilogue's disconnected term reads them)
      if (!g_dry && cudaStreamSynchronize(st) != cudaSuccess) {
        set_error("preparing tensor-core planes failed");
        r = LIBPT_ERR_CUDA;
        break;
      }
      for (OperandSet *set : {&p->L, &p->R})
        for (double **q : {&set->ovvv[0], &set->ovvv[1], &set->ovvv[2],
                           &set->ovvv[3], &set->oovo[0], &set->oovo[1],
                           &set->oovo[2], &set->oovo[3], &set->taup[0],
                           &set->taup[1]}) {
          if (!*q) continue;
          auto it = std::find(p->allocs.begin(), p->allocs.end(), (void *)*q);
          if (it != p->allocs.end()) {
            cudaFree(*q);
            p->allocs.erase(it);
          }
        }
    }
    if ((r = dalloc(p, (void **)&p->e_slot, (p->queue.size() + 1) * 8))) break;
    if (!g_dry &&
        cudaMemsetAsync(p->e_slot, 0, (p->queue.size() + 1) * 8, st) != cudaSuccess) {
      r = LIBPT_ERR_CUDA;
      break;
    }
    if ((r = dalloc(p, (void **)&p->d_err, sizeof(unsigned)))) break;
    if (!g_dry && cudaMemsetAsync(p->d_err, 0, sizeof(unsigned), st) != cudaSuccess) {
      r = LIBPT_ERR_CUDA;
      break;
    }
    // round geometry: the largest and smallest triples of the cases
    for (const SpinCase &c : p->cases)
      if (c.count) {
        p->ws_stride = std::max<int64_t>(p->ws_stride, c.ws_stride);
        p->ws_stride_min = p->ws_stride_min
                               ? std::min<int64_t>(p->ws_stride_min, c.ws_stride)
                               : c.ws_stride;
        p->ntiles_max = std::max(p->ntiles_max, c.ntiles);
        p->jobs_max = std::max(p->jobs_max, c.jobs.size());
      }
    if (p->ws_stride >= ((int64_t)1 << 31)) {
      // the epilogue indexes a triple's outputs with 32-bit offsets
      set_error("libpt_plan_create: orbital spaces too large (v > ~1000)");
      r = LIBPT_ERR_ARG;
      break;
    }
    if ((r = upload_views(p))) break;
    if (p->queue.empty()) break;
    if (p->arena) {
      // arena: size the batch buffers once, from what the arena has left
      const size_t d0 = Executor::bytes_for(0, p->jobs_max);
      const size_t per = (size_t)p->ws_stride * 8 +
                         (size_t)std::max(p->ntiles_max, 1) * 8 +
                         (Executor::bytes_for(1, p->jobs_max) - d0);
      const size_t used = (p->arena_used + 255) & ~size_t(255);
      const size_t slack = 3 * 256 + d0;
      const size_t left =
          p->arena_size > used + slack ? p->arena_size - used - slack : 0;
      // a requested round size is taken as is (the allocations below fail
      // if the arena cannot hold it); else as many triples as fit
      const size_t nb = std::min<size_t>(
          {arena_nb ? arena_nb : left / per, (size_t)4096, p->queue.size()});
      if (nb == 0) {
        set_error("scratch arena too small for one triple");
        r = LIBPT_ERR_NOMEM;
        break;
      }
      const size_t desc = Executor::bytes_for(nb, p->jobs_max);
      if ((r = dalloc(p, (void **)&p->ws, nb * p->ws_stride * 8))) break;
      if ((r = dalloc(p, (void **)&p->partials,
                      nb * std::max(p->ntiles_max, 1) * 8)))
        break;
      if ((r = dalloc(p, (void **)&p->d_desc, desc))) break;
      if ((r = p->exec.init(st, p->d_desc, desc, false))) break;
      p->exec_ready = true;
      p->ws_cap = (int64_t)nb * p->ws_stride;
      p->part_cap = (int64_t)nb * std::max(p->ntiles_max, 1);
      p->tri_cap = p->max_batch = nb;
      p->ws_budget = nb * p->ws_stride * 8;
      break;
    }
    // workspace budget: half of what is free, between 64 MiB and 16 GiB;
    // the buffers themselves are sized by the first run that needs them
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    p->ws_budget = std::min<size_t>(std::max<size_t>(fr / 2, (size_t)64 << 20),
                                    (size_t)16 << 30);
  } while (0);
  if (!r && !g_dry && profile_enabled()) {
    cudaStreamSynchronize(st);
    p->prof_prepare = wall_seconds() - t_start - p->prof_upload;
  }
  // deferred OVVV copies stay deferred only when nothing else in creation
  // reads them (the autotuner's probes would)
  if (!r && !p->deferred.empty() && tune_would_probe(p)) r = flush_deferred(p);
  const double t_tune = wall_seconds();
  if (!r && !g_dry && p->slices_auto) r = choose_slices(p);
  if (!r && !g_dry) r = autotune(p);
  p->prof_tune = wall_seconds() - t_tune;
  if (r) {
    plan_destroy(p);
    return r;
  }
  *out = p;
  return LIBPT_OK;
}

int plan_kernel_stats(libpt_plan *p, double *gemm_ms, int64_t *gemm_launches,
                      double *gemm_flops, double *epi_ms, int64_t *launches) {
  CK(cudaStreamSynchronize(p->st));
  double g = 0.0, e = 0.0, f = 0.0;
  ExecTiming &t = p->tm;
  for (size_t x = 0; x + 1 < t.ev_gemm.size(); x += 2) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, t.ev_gemm[x], t.ev_gemm[x + 1]));
    g += ms;
    CK(cudaEventElapsedTime(&ms, t.ev_epi[x], t.ev_epi[x + 1]));
    e += ms;
  }
  for (double v : t.flops) f += v;
  if (gemm_ms) *gemm_ms = g;
  if (gemm_launches) *gemm_launches = (int64_t)(t.ev_gemm.size() / 2);
  if (gemm_flops) *gemm_flops = f;
  if (epi_ms) *epi_ms = e;
  if (launches) *launches = p->launches;
  t.clear();
  p->launches = 0;
  return LIBPT_OK;
}

size_t plan_footprint(int kind, size_t oa, size_t va, size_t ob, size_t vb,
                      int dtype, int precision, bool host, size_t nb) {
  // a sizing pass over a fake, 256-byte aligned arena of unbounded size
  static const double dummy = 0.0;
  const void *args[10];
  for (int a = 0; a < 10; ++a) args[a] = &dummy;
  char *const fake = reinterpret_cast<char *>((uintptr_t)1 << 44);
  libpt_plan *p = nullptr;
  g_dry = true;
  const int r = plan_create(kind, oa, va, ob, vb, args, dtype, precision, host,
                            nullptr, &p, fake, (size_t)1 << 60, nb);
  g_dry = false;
  if (r || !p) return 0;
  const size_t used = p->arena_used;
  plan_destroy(p);
  return ((used + 255) & ~size_t(255)) + 256;   // + alignment of the base
}

void plan_destroy(libpt_plan *p) {
  if (!p) return;
  if (p->st) cudaStreamSynchronize(p->st);
  if (p->st_up) {
    cudaStreamSynchronize(p->st_up);
    cudaStreamDestroy(p->st_up);
  }
  if (p->ev_up) cudaEventDestroy(p->ev_up);
  p->tm.clear();
  if (p->exec_ready) p->exec.destroy();
  for (void *a : p->allocs) cudaFree(a);
  delete p;
}

double plan_flops(const libpt_plan *p, int64_t first, int64_t n) {
  double f = 0.0;
  for (const SpinCase &c : p->cases) {
    const int64_t lo = std::max(first, c.first);
    const int64_t hi = std::min(first + n, c.first + c.count);
    if (hi > lo) f += (double)(hi - lo) * c.flops_per_triple;
  }
  return f;
}

}  // namespace ptb
