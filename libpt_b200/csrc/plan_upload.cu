// Device memory of a plan and the uploads of the caller's arrays: arena or
// cudaMalloc allocations, the page-locked staging ring and host copy pool,
// the padded operand blocks, and the restricted FP64 host-array solve that
// streams its OVVV rows by occupied index beside the triples.
// Part of the triples engine (plan_*.cu); internal declarations shared by
// those files are in plan_impl.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "plan_impl.h"
#include <condition_variable>
#include <mutex>
#include <thread>

namespace ptb {

int dalloc(libpt_plan *p, void **ptr, size_t bytes) {
  *ptr = nullptr;
  if (bytes == 0) bytes = 256;
  if (p->arena) {   // carve from the caller's arena; never freed
    const size_t off = (p->arena_used + 255) & ~size_t(255);
    if (off + bytes > p->arena_size) {
      set_error("scratch arena exhausted (" + std::to_string(off + bytes) +
                " of " + std::to_string(p->arena_size) + " bytes)");
      return LIBPT_ERR_NOMEM;
    }
    *ptr = p->arena + off;
    p->arena_used = off + bytes;
    return LIBPT_OK;
  }
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) {
    set_error("cudaMalloc(" + std::to_string(bytes) +
              " bytes): " + cudaGetErrorString(e));
    cudaGetLastError();
    return LIBPT_ERR_NOMEM;
  }
  p->allocs.push_back(*ptr);
  return LIBPT_OK;
}

PinnedRing &pinned_ring() {
  static PinnedRing r;
  return r;
}

// Host copies with up to 8 threads (large chunks only): a pool of worker
// threads started on first use and kept for the life of the process (it is
// never destroyed, so no worker outlives its state at exit).
class CopyPool {
 public:
  static CopyPool &get() {
    static CopyPool *pool = new CopyPool();
    return *pool;
  }

  void copy(void *dst, const void *src, size_t n) {
    if (n < ((size_t)8 << 20) || nw_ == 0) {
      std::memcpy(dst, src, n);
      return;
    }
    std::lock_guard<std::mutex> one_at_a_time(submit_mu_);
    const size_t per = (n / (nw_ + 1) + 4095) & ~(size_t)4095;
    {
      std::lock_guard<std::mutex> g(mu_);
      dst_ = static_cast<char *>(dst);
      src_ = static_cast<const char *>(src);
      n_ = n;
      per_ = per;
      pending_ = nw_;
      ++gen_;
    }
    work_cv_.notify_all();
    std::memcpy(dst, src, std::min(per, n));   // part 0 on this thread
    std::unique_lock<std::mutex> g(mu_);
    done_cv_.wait(g, [&] { return pending_ == 0; });
  }

 private:
  CopyPool() {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned want = std::min(8u, hw) - 1;
    for (unsigned t = 1; t <= want; ++t) {
      try {
        std::thread([this, t] { work(t); }).detach();
        nw_ = t;
      } catch (...) {
        break;
      }
    }
  }

  void work(unsigned t) {
    uint64_t seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> g(mu_);
      work_cv_.wait(g, [&] { return gen_ != seen; });
      seen = gen_;
      char *d = dst_;
      const char *s = src_;
      const size_t n = n_, o = (size_t)t * per_, len = per_;
      g.unlock();
      if (o < n) std::memcpy(d + o, s + o, std::min(len, n - o));
      g.lock();
      if (--pending_ == 0) done_cv_.notify_one();
    }
  }

  unsigned nw_ = 0;   // workers; part t of a copy goes to worker t
  std::mutex submit_mu_, mu_;
  std::condition_variable work_cv_, done_cv_;
  uint64_t gen_ = 0;
  unsigned pending_ = 0;
  char *dst_ = nullptr;
  const char *src_ = nullptr;
  size_t n_ = 0, per_ = 0;
};

void par_memcpy(void *dst, const void *src, size_t n) {
  CopyPool::get().copy(dst, src, n);
}

// Upload one amplitude + integrals set into padded blocks.
int upload_set(libpt_plan *p, Uploader &up, const Sizes &S, OperandSet &set,
               const void *tau, const void *oovo, const void *ovvv) {
  const int nb = p->unrestricted ? 4 : 2;
  const size_t es = p->dtype ? 4 : 8;
  int64_t off_t = 0, off_o = 0, off_v = 0;
  for (int b = 0; b < nb; ++b) {
    int64_t rows, w;
    S.tau_shape(b, rows, w);
    if (dalloc(p, (void **)&set.tau[b], rows * pad4(w) * 8)) return LIBPT_ERR_NOMEM;
    if (int r = up.put(set.tau[b], (const char *)tau + off_t * es, rows, w, pad4(w)))
      return r;
    off_t += S.oovv(b);
    S.oovo_shape(b, rows, w);
    if (dalloc(p, (void **)&set.oovo[b], rows * pad4(w) * 8)) return LIBPT_ERR_NOMEM;
    if (int r = up.put(set.oovo[b], (const char *)oovo + off_o * es, rows, w, pad4(w)))
      return r;
    off_o += S.oovo(b);
    S.ovvv_shape(b, rows, w);
    if (p->precision == LIBPT_PREC_EMU64 && !up.host && !up.fp32) {
      // sliced in place from the caller's device block: no FP64 copy
      set.ovvv_src[b] = (const double *)ovvv + off_v;
    } else {
      if (dalloc(p, (void **)&set.ovvv[b], rows * pad4(w) * 8))
        return LIBPT_ERR_NOMEM;
      if (p->defer_ovvv) {   // restricted: the first index is occupied
        p->deferred.push_back({set.ovvv[b], (const char *)ovvv + off_v * es,
                               rows / p->oa, w, pad4(w)});
      } else if (int r = up.put(set.ovvv[b], (const char *)ovvv + off_v * es,
                                rows, w, pad4(w))) {
        return r;
      }
    }
    off_v += S.ovvv(b);
  }
  if (!p->unrestricted) {   // src/pt.c:471-473: baba blocks alias abab
    set.tau[3] = set.tau[1];
    set.oovo[3] = set.oovo[1];
    set.ovvv[3] = set.ovvv[1];
    set.ovvv_src[3] = set.ovvv_src[1];
  }
  // packed-pair copies of the same-spin amplitudes
  for (int s = 0; s < (p->unrestricted ? 2 : 1); ++s) {
    const int64_t o = s ? S.ob : S.oa, v = s ? S.vb : S.va;
    const int64_t ldp = pad4(npair(v));
    if (dalloc(p, (void **)&set.taup[s], o * o * ldp * 8)) return LIBPT_ERR_NOMEM;
    DEV(pack_pairs_launch(set.tau[s ? 2 : 0], set.taup[s], o * o, (int)v,
                         pad4(v), ldp, p->st));
  }
  return LIBPT_OK;
}

// Makes every deferred OVVV copy now (on the plan's stream).
int flush_deferred(libpt_plan *p) {
  Uploader up{p, true, p->dtype == 1};
  up.stage[0] = p->up_stage[0];
  up.stage[1] = p->up_stage[1];
  up.stage_bytes = p->up_stage_bytes;
  for (const DeferredBlock &d : p->deferred)
    if (int r = up.put(d.dst, d.src, d.rows_per_index * p->oa, d.w, d.dpitch))
      return r;
  p->deferred.clear();
  return LIBPT_OK;
}

int plan_run_streamed(libpt_plan *p) {
  const size_t total = p->queue.size();
  if (p->deferred.empty()) return plan_run(p, nullptr, total);
  if (g_dry) return LIBPT_OK;
  // triples by the largest occupied index they read (every OVVV row a
  // triple (i, j, k) reads belongs to i, j or k)
  const int o = p->oa;
  std::vector<std::vector<int64_t>> by_index((size_t)o);
  std::vector<int64_t> all(total);
  for (size_t q = 0; q < total; ++q) {
    const int4 t = p->queue[q];
    by_index[(size_t)std::max(t.y, std::max(t.z, t.w))].push_back((int64_t)q);
    all[q] = (int64_t)q;
  }
  // round resources for the whole queue first: growing them later would
  // wait for the triples already running
  if (int r = ensure_capacity(p, all)) return r;
  if (!p->st_up) {
    CK(cudaStreamCreateWithFlags(&p->st_up, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&p->ev_up, cudaEventDisableTiming));
  }
  Uploader up{p, true, p->dtype == 1};
  up.stage[0] = p->up_stage[0];
  up.stage[1] = p->up_stage[1];
  up.stage_bytes = p->up_stage_bytes;
  up.s = p->st_up;
  // the copies start after everything plan creation queued on its stream
  CK(cudaEventRecord(p->ev_up, p->st));
  CK(cudaStreamWaitEvent(p->st_up, p->ev_up, 0));
  const size_t es = p->dtype ? 4 : 8;
  for (int m = 0; m < o; ++m) {
    for (const DeferredBlock &d : p->deferred) {
      const int64_t r0 = (int64_t)m * d.rows_per_index;
      if (int r = up.put(d.dst + r0 * d.dpitch, d.src + (size_t)(r0 * d.w) * es,
                         d.rows_per_index, d.w, d.dpitch))
        return r;
    }
    CK(cudaEventRecord(p->ev_up, p->st_up));
    CK(cudaStreamWaitEvent(p->st, p->ev_up, 0));
    if (!by_index[(size_t)m].empty())
      if (int r = run_entries(p, by_index[(size_t)m])) return r;
  }
  p->deferred.clear();
  return LIBPT_OK;
}

}  // namespace ptb
