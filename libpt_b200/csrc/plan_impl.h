// Internal declarations shared by the parts of the triples engine
// (plan.cu, plan_views.cu, plan_upload.cu, plan_cases.cu, plan_emu.cu,
// plan_tune.cu, plan_run.cu).  Not part of the library's interface.
#pragma once

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "plan.h"
#include "tune.h"

namespace ptb {

// Sizing pass (plan_footprint): plan creation runs its host logic with
// device allocations carved from a fake arena and every device operation
// skipped, so the arena's high-water mark is the plan's exact footprint.
extern thread_local bool g_dry;

// A device operation of plan creation: skipped in the sizing pass.
#define DEV(call)                                                          \
  do {                                                                     \
    if (!::ptb::g_dry) CK(call);                                           \
  } while (0)

inline int64_t pad4(int64_t x) { return (x + 3) & ~int64_t(3); }
inline int64_t pad32(int64_t x) { return (x + 31) & ~int64_t(31); }
inline int64_t npair(int64_t v) { return v * (v - 1) / 2; }
inline int ksteps(int64_t k) { return (int)((k + GEMM_BK - 1) / GEMM_BK); }

// ---- tensor-map views (plan_views.cu) ---------------------------------------
// A-view of a padded block [P][Q][R][Kpad] with logical K: dims (K, R, Q, P),
// box (4, bm, 1, 1); B-view of a padded block [P][K][Nld] with logical N:
// dims (N, K, P), box (4, GEMM_BK, 1).
int map_a(CUtensorMap *m, const double *p, int64_t K, int64_t R, int64_t Q,
          int64_t P, int bm);
int map_b(CUtensorMap *m, const double *p, int64_t N, int64_t Nld, int64_t K,
          int64_t P);
// Tensor-core views of a case: TF32 plane pairs at map indices 2i, 2i+1.
int build_tc(libpt_plan *p, SpinCase &c);

// ---- device memory and uploads (plan_upload.cu) -----------------------------
// A device buffer of the plan: carved from its arena, or cudaMalloc'd and
// freed with the plan.
int dalloc(libpt_plan *p, void **ptr, size_t bytes);

// Page-locked staging for host uploads, shared by the process: two 64 MiB
// buffers used in turn, so the host copy of one chunk into page-locked
// memory overlaps the DMA of the previous one (pageable cudaMemcpyAsync
// copies through the driver's own small buffers, synchronously).
struct PinnedRing {
  std::mutex mu;   // one upload uses the ring at a time
  char *buf[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  bool tried = false, ok = false;
  static constexpr size_t BYTES = (size_t)64 << 20;
  bool ready() {   // with mu held
    if (tried) return ok;
    tried = true;
    ok = true;
    for (int b = 0; b < 2 && ok; ++b)
      ok = cudaHostAlloc((void **)&buf[b], BYTES, cudaHostAllocDefault) ==
               cudaSuccess &&
           cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming) ==
               cudaSuccess;
    if (!ok) cudaGetLastError();
    return ok;
  }
};
PinnedRing &pinned_ring();
// Host copy with up to 8 threads (large copies only).
void par_memcpy(void *dst, const void *src, size_t n);

// Copies rows x w elements (FP64 or FP32, host or device) into a padded FP64
// device block rows x dpitch.  Host sources go through page-locked and
// device staging buffers in chunks of whole rows (two of each, used in
// turn), device sources are repacked directly.
struct Uploader {
  libpt_plan *p;
  bool host, fp32;
  size_t stage_cap = PinnedRing::BYTES;   // per staging buffer
  void *stage[2] = {nullptr, nullptr};    // device staging
  size_t stage_bytes = 0;
  int slot = 0;
  cudaStream_t s = nullptr;               // copy stream (null: the plan's)

  int put(double *dst, const void *src, int64_t rows, int64_t w,
          int64_t dpitch) {
    if (rows <= 0 || dpitch <= 0) return LIBPT_OK;
    const size_t es = fp32 ? 4 : 8;
    const cudaStream_t cs = s ? s : p->st;
    if (!host) {
      if (w == dpitch && !fp32)
        DEV(cudaMemcpyAsync(dst, src, (size_t)rows * w * 8,
                            cudaMemcpyDeviceToDevice, cs));
      else
        DEV(repack_launch(src, fp32, dst, rows, w, dpitch, cs));
      return LIBPT_OK;
    }
    if (!stage[0]) {
      stage_bytes = stage_cap;
      if (dalloc(p, &stage[0], stage_bytes) || dalloc(p, &stage[1], stage_bytes))
        return LIBPT_ERR_NOMEM;
    }
    if (g_dry) return LIBPT_OK;
    // chunks: whole rows (a flat run of elements when unpadded)
    const bool flat = w == dpitch;
    const int64_t unit = flat ? 1 : std::max<int64_t>(w, 1);
    const int64_t total = flat ? rows * w : rows;
    const int64_t chunk =
        std::max<int64_t>(1, (int64_t)(stage_bytes / (es * unit)));
    PinnedRing &ring = pinned_ring();
    std::lock_guard<std::mutex> lk(ring.mu);
    const bool pinned = ring.ready();
    for (int64_t x0 = 0; x0 < total; x0 += chunk) {
      const int64_t nx = std::min(chunk, total - x0);
      const size_t bytes = (size_t)(nx * unit) * es;
      const char *from = (const char *)src + (size_t)(x0 * unit) * es;
      void *dstage = stage[slot];
      if (pinned) {
        CK(cudaEventSynchronize(ring.done[slot]));   // its last DMA is done
        par_memcpy(ring.buf[slot], from, bytes);
        CK(cudaMemcpyAsync(dstage, ring.buf[slot], bytes,
                           cudaMemcpyHostToDevice, cs));
        CK(cudaEventRecord(ring.done[slot], cs));
      } else {
        CK(cudaMemcpyAsync(dstage, from, bytes, cudaMemcpyHostToDevice, cs));
      }
      if (flat)
        CK(repack_launch(dstage, fp32, dst + x0, 1, nx, nx, cs));
      else
        CK(repack_launch(dstage, fp32, dst + x0 * dpitch, nx, w, dpitch,
                         cs));
      slot ^= 1;
    }
    // the ring's buffers may be reused by the next upload only after these
    // DMAs: each slot's event covers its last copy
    return LIBPT_OK;
  }
};

// Element counts of the four spin blocks of each tensor family.
struct Sizes {
  int64_t oa, va, ob, vb;
  int64_t oovv(int b) const {
    return b == 0 ? oa * oa * va * va : b == 1 ? oa * ob * va * vb
         : b == 2 ? ob * ob * vb * vb : ob * oa * vb * va;
  }
  int64_t oovo(int b) const {
    return b == 0 ? oa * oa * va * oa : b == 1 ? oa * ob * va * ob
         : b == 2 ? ob * ob * vb * ob : ob * oa * vb * oa;
  }
  int64_t ovvv(int b) const {
    return b == 0 ? oa * va * npair(va) : b == 1 ? oa * vb * va * vb
         : b == 2 ? ob * vb * npair(vb) : ob * va * vb * va;
  }
  // (rows, inner width) of each block in pt.h layout
  void tau_shape(int b, int64_t &rows, int64_t &w) const {
    rows = b == 0 ? oa * oa * va : b == 1 ? oa * ob * va
         : b == 2 ? ob * ob * vb : ob * oa * vb;
    w = (b == 0 || b == 3) ? va : vb;
  }
  void oovo_shape(int b, int64_t &rows, int64_t &w) const {
    rows = b == 0 ? oa * oa * va : b == 1 ? oa * ob * va
         : b == 2 ? ob * ob * vb : ob * oa * vb;
    w = (b == 0 || b == 3) ? oa : ob;
  }
  void ovvv_shape(int b, int64_t &rows, int64_t &w) const {
    rows = b == 0 ? oa * va : b == 1 ? oa * vb * va
         : b == 2 ? ob * vb : ob * va * vb;
    w = b == 0 ? npair(va) : b == 1 ? vb : b == 2 ? npair(vb) : va;
  }
};

// Upload one amplitude + integrals set into padded blocks.
int upload_set(libpt_plan *p, Uploader &up, const Sizes &S, OperandSet &set,
               const void *tau, const void *oovo, const void *ovvv);
// Makes every deferred OVVV copy now (on the plan's stream).
int flush_deferred(libpt_plan *p);

// ---- spin cases, job templates, queue (plan_cases.cu) -----------------------
int add_cases(libpt_plan *p);
// Copies each case's kernel views (tensor maps) and epilogue arguments to
// device memory, where the kernels read them.  Re-run after any map change.
int upload_views(libpt_plan *p);

// ---- emulated FP64 operands (plan_emu.cu) -----------------------------------
int i8_maxima(libpt_plan *p);
int i8_exponents(libpt_plan *p);
int i8_encode(libpt_plan *p, SpinCase &c);
int i8_planes(libpt_plan *p, SpinCase &c);
int choose_digits(libpt_plan *p);
int choose_slices(libpt_plan *p);

// ---- autotuner (plan_tune.cu) -----------------------------------------------
bool tune_would_probe(libpt_plan *p);
int autotune(libpt_plan *p);

// ---- rounds (plan_run.cu) ---------------------------------------------------
// Sizes the round resources for `ents` (up to the workspace budget).
int ensure_capacity(libpt_plan *p, const std::vector<int64_t> &ents);
// Runs queue entries in rounds, each filling the plan's round resources.
int run_entries(libpt_plan *p, const std::vector<int64_t> &ents);

}  // namespace ptb
