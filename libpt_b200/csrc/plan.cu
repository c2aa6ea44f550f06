// The triples engine: operand preparation, spin cases, job templates and the
// batched run over the triples queue.
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

#include "plan.h"
#include "tune.h"
#include "pt.h"

namespace ptb {

static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }

// Sizing pass (plan_footprint): plan creation runs its host logic with
// device allocations carved from a fake arena and every device operation
// skipped, so the arena's high-water mark is the plan's exact footprint.
static thread_local bool g_dry = false;

// A device operation of plan creation: skipped in the sizing pass.
#define DEV(call)                                                          \
  do {                                                                     \
    if (!g_dry) CK(call);                                                  \
  } while (0)
const char *last_error() { return g_last_error.c_str(); }

namespace {

int64_t pad4(int64_t x) { return (x + 3) & ~int64_t(3); }
int64_t pad32(int64_t x) { return (x + 31) & ~int64_t(31); }
int64_t npair(int64_t v) { return v * (v - 1) / 2; }
int ksteps(int64_t k) { return (int)((k + GEMM_BK - 1) / GEMM_BK); }


typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType,
                                  cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p,
                                cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// A-view of a padded block [P][Q][R][Kpad] with logical K: dims (K, R, Q, P),
// box (4, bm, 1, 1).
int map_a(CUtensorMap *m, const double *p, int64_t K, int64_t R, int64_t Q,
          int64_t P, int bm) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  const int64_t kp = pad4(K);
  cuuint64_t dims[4] = {(cuuint64_t)std::max<int64_t>(K, 1),
                        (cuuint64_t)std::max<int64_t>(R, 1),
                        (cuuint64_t)std::max<int64_t>(Q, 1),
                        (cuuint64_t)std::max<int64_t>(P, 1)};
  cuuint64_t strides[3] = {(cuuint64_t)(kp * 8), (cuuint64_t)(R * kp * 8),
                           (cuuint64_t)(Q * R * kp * 8)};
  cuuint32_t box[4] = {4, (cuuint32_t)bm, 1, 1};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)p, dims,
                   strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (A view) failed: " + std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

// B-view of a padded block [P][K][Nld] with logical N: dims (N, K, P),
// box (4, GEMM_BK, 1).
int map_b(CUtensorMap *m, const double *p, int64_t N, int64_t Nld, int64_t K,
          int64_t P) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  cuuint64_t dims[3] = {(cuuint64_t)std::max<int64_t>(N, 1),
                        (cuuint64_t)std::max<int64_t>(K, 1),
                        (cuuint64_t)std::max<int64_t>(P, 1)};
  cuuint64_t strides[2] = {(cuuint64_t)(Nld * 8), (cuuint64_t)(K * Nld * 8)};
  cuuint32_t box[3] = {4, (cuuint32_t)GEMM_BK, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)p, dims,
                   strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (B view) failed: " + std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

int tc_encode(CUtensorMap *m, const float *p, int rank, const cuuint64_t *dims,
              const cuuint64_t *strides, const cuuint32_t *box) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, (void *)p, dims,
                   strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (tensor-core view) failed: " +
              std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

int dalloc(libpt_plan *p, void **ptr, size_t bytes);

}  // namespace

// Digit-plane views (see slice_a / slice_b): 32-byte K chunks of rows
// stored contiguously, boxes of 32 bytes x 128 (A) or bn (B) rows swizzled
// to 32 bytes.  A: (32, R, nK, Q*P, 2S); B: (32, N, nK, P, S).
int i8_map_a(CUtensorMap *m, const signed char *p, int64_t K, int64_t R,
             int64_t Q, int64_t P, int S) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  constexpr int W = I8_KCHUNK;
  const int64_t kpi = i8_kpad(K), nk = kpi / W, npq = Q * P;
  cuuint64_t dims[5] = {W, (cuuint64_t)R, (cuuint64_t)nk, (cuuint64_t)npq,
                        (cuuint64_t)(2 * S)};
  cuuint64_t str[4] = {W, (cuuint64_t)(R * W), (cuuint64_t)(R * kpi),
                       (cuuint64_t)(npq * R * kpi)};
  cuuint32_t box[5] = {W, (cuuint32_t)TC_BM, 1, 1, 1};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, (void *)p, dims, str,
                   box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (INT8 A view) failed: " +
              std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

int i8_map_b(CUtensorMap *m, const signed char *p, int64_t K, int64_t N,
             int64_t P, int S, int bn) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  constexpr int W = I8_KCHUNK;
  const int64_t kpi = i8_kpad(K), nk = kpi / W;
  cuuint64_t dims[5] = {W, (cuuint64_t)N, (cuuint64_t)nk, (cuuint64_t)P,
                        (cuuint64_t)S};
  cuuint64_t str[4] = {W, (cuuint64_t)(N * W), (cuuint64_t)(N * kpi),
                       (cuuint64_t)(P * N * kpi)};
  cuuint32_t box[5] = {W, (cuuint32_t)bn, 1, 1, 1};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, (void *)p, dims, str,
                   box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (INT8 B view) failed: " +
              std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

int dmma_map_a(CUtensorMap *m, const double *p, int64_t K, int64_t R,
               int64_t Q, int64_t P, int bm) {
  return map_a(m, p, K, R, Q, P, bm);
}

int dmma_map_b(CUtensorMap *m, const double *p, int64_t N, int64_t Nld,
               int64_t K, int64_t P) {
  return map_b(m, p, N, Nld, K, P);
}

int tc_map_a(CUtensorMap *m, const float *p, int64_t K, int64_t R, int64_t Q,
             int64_t P) {
  const int64_t kp = pad4(K);
  cuuint64_t dims[4] = {(cuuint64_t)std::max<int64_t>(K, 1),
                        (cuuint64_t)std::max<int64_t>(R, 1),
                        (cuuint64_t)std::max<int64_t>(Q, 1),
                        (cuuint64_t)std::max<int64_t>(P, 1)};
  cuuint64_t strides[3] = {(cuuint64_t)(kp * 4), (cuuint64_t)(R * kp * 4),
                           (cuuint64_t)(Q * R * kp * 4)};
  cuuint32_t box[4] = {(cuuint32_t)tc_kchunk_elems(TC_TF32), (cuuint32_t)TC_BM,
                       1, 1};
  return tc_encode(m, p, 4, dims, strides, box);
}

int tc_map_b(CUtensorMap *m, const float *p, int64_t K, int64_t N, int64_t P) {
  const int64_t kp = pad4(K);
  cuuint64_t dims[3] = {(cuuint64_t)std::max<int64_t>(K, 1),
                        (cuuint64_t)std::max<int64_t>(N, 1),
                        (cuuint64_t)std::max<int64_t>(P, 1)};
  cuuint64_t strides[2] = {(cuuint64_t)(kp * 4), (cuuint64_t)(N * kp * 4)};
  cuuint32_t box[3] = {(cuuint32_t)tc_kchunk_elems(TC_TF32), (cuuint32_t)TC_BN,
                       1};
  return tc_encode(m, p, 3, dims, strides, box);
}

namespace {

// TF32 planes of an operand, made once per (source block, role).
int get_planes(libpt_plan *p, const OpDesc &d, Planes *out) {
  const std::pair<const double *, int> key(d.src, d.role);
  for (auto &e : p->planes)
    if (e.first == key) {
      *out = e.second;
      return LIBPT_OK;
    }
  Planes pl;
  const int64_t kp = pad4(d.K);
  if (d.role == 0) {
    const int64_t n = d.P * d.Q * d.R * kp;
    if (dalloc(p, (void **)&pl.hi, n * 4) || dalloc(p, (void **)&pl.lo, n * 4))
      return LIBPT_ERR_NOMEM;
    DEV(split_tf32_launch(d.src, pl.hi, pl.lo, n, p->st));
  } else {
    const int64_t n = d.P * d.N * kp;
    if (dalloc(p, (void **)&pl.hi, n * 4) || dalloc(p, (void **)&pl.lo, n * 4))
      return LIBPT_ERR_NOMEM;
    DEV(transpose_split_tf32_launch(d.src, pl.hi, pl.lo, d.P, (int)d.K, d.N,
                                   d.Nld, kp, p->st));
  }
  p->planes.push_back({key, pl});
  *out = pl;
  return LIBPT_OK;
}

// Tensor-core views of a case: plane pairs at map indices 2i, 2i+1.
int build_tc(libpt_plan *p, SpinCase &c) {
  for (int i = 0; i < MAX_MAPS; ++i) {
    const OpDesc &d = c.opd[i];
    if (d.role < 0) continue;
    if (2 * i + 1 >= TC_MAX_MAPS) {
      set_error("too many tensor-core operand views");
      return LIBPT_ERR_ARG;
    }
    Planes pl;
    if (int r = get_planes(p, d, &pl)) return r;
    for (int h = 0; h < 2; ++h) {
      const float *pp = h ? pl.lo : pl.hi;
      int r = d.role == 0 ? tc_map_a(&c.tcmaps.m[2 * i + h], pp, d.K, d.R, d.Q, d.P)
                          : tc_map_b(&c.tcmaps.m[2 * i + h], pp, d.K, d.N, d.P);
      if (r) return r;
    }
  }
  return LIBPT_OK;
}

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

SegT seg(int amap, int bmap, bool neg, int aq, int ap, int bp, int64_t k) {
  SegT s;
  s.amap = (int16_t)amap;
  s.bmap = (int16_t)bmap;
  s.neg = neg ? 1 : 0;
  s.aq = (int8_t)aq;
  s.ap = (int8_t)ap;
  s.bp = (int8_t)bp;
  s.ksteps = ksteps(k);
  s.k = (int32_t)k;
  return s;
}

enum { I = 0, J = 1, K = 2 };

// Encode a DMMA view (FP64 path) and remember what it views, for the
// tensor-core paths; fam/part classify the operand for emulated FP64.
int reg_a(libpt_plan *p, SpinCase &c, int idx, const double *ptr, int64_t Kd,
          int64_t R, int64_t Q, int64_t P, int fam, int part) {
  OpDesc &d = c.opd[idx];
  d.role = 0;
  d.src = ptr;
  d.K = Kd;
  d.R = R;
  d.Q = Q;
  d.P = P;
  d.fam = fam;
  d.part = part;
  if (p->precision != LIBPT_PREC_FP64) return LIBPT_OK;
  return map_a(&c.maps.m[idx], ptr, Kd, R, Q, P, c.bm);
}

// B operand [P][K][N] in the engine's padded layout (row length Nld), or --
// when src_w > 0 -- the caller's unpadded pt.h block whose N index is
// row-padded: n = y*src_w + c, c < src_wsrc real, rows of src_ld elements.
int reg_b(libpt_plan *p, SpinCase &c, int idx, const double *ptr, int64_t N,
          int64_t Nld, int64_t Kd, int64_t P, int fam, int part,
          int64_t src_ld = 0, int64_t src_w = 0, int64_t src_wsrc = 0) {
  OpDesc &d = c.opd[idx];
  d.role = 1;
  d.src = ptr;
  d.K = Kd;
  d.N = N;
  d.Nld = Nld;
  d.P = P;
  d.fam = fam;
  d.part = part;
  if (src_w > 0) {
    d.ldsrc = src_ld;
    d.w = src_w;
    d.wsrc = src_wsrc;
  } else {
    d.ldsrc = Nld;
    d.w = Nld;
    d.wsrc = Nld;
  }
  if (p->precision != LIBPT_PREC_FP64) return LIBPT_OK;
  return map_b(&c.maps.m[idx], ptr, N, Nld, Kd, P);
}

// Scale families of emulated FP64: the A operands of a job (amplitude and
// OOVO blocks of one spin-block index) and its B operands (OVVV block and
// the amplitude block of the same index) share row / column scales.
int fam_a(const libpt_plan *p, int set, int b) {
  return set * 8 + (!p->unrestricted && b == 3 ? 1 : b);
}
int fam_b(const libpt_plan *p, int set, int b) {
  return 100 + set * 8 + (!p->unrestricted && b == 3 ? 1 : b);
}

// OVVV block b of a set as a B operand: the padded FP64 copy, or the
// caller's pt.h block when it is sliced in place (emulated FP64, device
// inputs).  N counts the padded-convention columns.
int reg_ovvv(libpt_plan *p, SpinCase &c, int idx, const OperandSet &S, int b,
             int64_t N, int64_t Nld, int64_t Kd, int64_t P, int fam) {
  if (S.ovvv[b])
    return reg_b(p, c, idx, S.ovvv[b], N, Nld, Kd, P, fam, 0);
  const int64_t va = p->va, vb = p->vb;
  int64_t ld, w, wsrc;
  if (b == 0 || b == 2) {   // packed pairs: no inner padding
    const int64_t v = b ? vb : va;
    ld = w = wsrc = v * (v - 1) / 2;
  } else if (b == 1) {      // [oa][vb][va][vb]: N = (y < va, c < vb)
    ld = va * vb;
    w = pad4(vb);
    wsrc = vb;
  } else {                  // [ob][va][vb][va]
    ld = vb * va;
    w = pad4(va);
    wsrc = va;
  }
  return reg_b(p, c, idx, S.ovvv_src[b], N, Nld, Kd, P, fam, 0, ld, w, wsrc);
}

// Same-spin case: four maps per operand set, one job (T) per set.
int build_aaa(libpt_plan *p, SpinCase &c) {
  const int s = c.flip;
  const int64_t o = c.oa, v = c.va, np = npair(v), ldT = pad4(np);
  const int nset = p->ft ? 2 : 1;
  int64_t offs[2];
  int64_t stride = 0;
  for (int x = 0; x < nset; ++x) {
    offs[x] = stride;
    stride += pad32(v * ldT);
  }
  for (int x = 0; x < nset; ++x) {
    const OperandSet &set = x ? p->R : p->L;
    const int b0 = 4 * x;
    const int bi = s ? 2 : 0;
    const int fa = fam_a(p, x, bi), fb = fam_b(p, x, bi);
    if (int r = reg_a(p, c, b0 + 0, set.tau[bi], v, v, o, o, fa, 0)) return r;
    if (int r = reg_a(p, c, b0 + 1, set.oovo[bi], o, v, o, o, fa, 1)) return r;
    if (int r = reg_ovvv(p, c, b0 + 2, set, bi, np, ldT, v, o, fb)) return r;
    if (int r = reg_b(p, c, b0 + 3, set.taup[s], np, ldT, o, o, fb, 1)) return r;
    JobT j;
    j.off = offs[x];
    j.M = (int)v;
    j.N = (int)ldT;
    j.ldc = ldT;
    j.nseg = 6;
    // T[x][pair] = sum_d (t_ij - t_ik - t_kj)[x][d] I_(k,j,i)[d][pair]
    //            + sum_l (O_jk - O_ik - O_ji)[x][l] tp_(i,j,k)[l][pair]
    j.seg[0] = seg(b0 + 0, b0 + 2, false, J, I, K, v);
    j.seg[1] = seg(b0 + 0, b0 + 2, true, K, I, J, v);
    j.seg[2] = seg(b0 + 0, b0 + 2, true, J, K, I, v);
    j.seg[3] = seg(b0 + 1, b0 + 3, false, K, J, I, o);
    j.seg[4] = seg(b0 + 1, b0 + 3, true, K, I, J, o);
    j.seg[5] = seg(b0 + 1, b0 + 3, true, I, J, K, o);
    if (np > 0) c.jobs.push_back(j);
  }
  EpiArgs &e = c.epi;
  memset(&e, 0, sizeof(e));
  c.ws_stride = stride;
  e.offL[0] = offs[0];
  e.offR[0] = p->ft ? offs[1] : -1;
  e.ld[0] = ldT;
  e.oa = (int)o;
  e.va = (int)v;
  e.ob = (int)o;
  e.vb = (int)v;
  const int64_t ovoff = s ? (int64_t)p->oa * p->va : 0;
  e.d_a = p->d_ov + ovoff;
  e.ov1_a = p->ov1 + ovoff;
  e.ov2_a = p->ov2 + ovoff;
  e.g1_aa = p->oovv[s ? 2 : 0];
  e.g1_ld_aa = v;
  e.g2_aa = p->L.tau[s ? 2 : 0];
  e.g2_ld_aa = pad4(v);
  // tiles (a0, b0, c0) holding at least one a > b > c
  std::vector<int4> tiles;
  for (int64_t a0 = 0; a0 < v; a0 += EPI_A) {
    const int64_t amax = std::min<int64_t>(a0 + EPI_A - 1, v - 1);
    for (int64_t b0 = 0; b0 <= a0; b0 += EPI_B) {
      if (amax - 1 < b0) continue;
      const int64_t bmax = std::min<int64_t>(b0 + EPI_B - 1, amax - 1);
      for (int64_t c0 = 0; c0 < bmax; c0 += EPI_C)
        tiles.push_back(make_int4((int)a0, (int)b0, (int)c0, 0));
    }
  }
  c.ntiles = (int)tiles.size();
  c.ctiles = 1;
  if (c.ntiles) {
    if (dalloc(p, (void **)&c.d_tiles, tiles.size() * sizeof(int4))) return LIBPT_ERR_NOMEM;
    DEV(cudaMemcpyAsync(c.d_tiles, tiles.data(), tiles.size() * sizeof(int4),
                       cudaMemcpyHostToDevice, p->st));
    DEV(cudaStreamSynchronize(p->st));
  }
  e.ntiles = c.ntiles;
  e.tiles = c.d_tiles;
  e.ctiles = c.ctiles;
  e.has_f = p->has_f ? 1 : 0;
  const double vv = (double)v;
  c.flops_per_triple = 3.0 * vv * vv * vv * (vv - 1) + 6.0 * o * vv * vv * vv;
  if (p->ft) c.flops_per_triple *= 2;
  return LIBPT_OK;
}

// Mixed-spin case: twelve maps per operand set, three jobs (U1, U2, P).
int build_aab(libpt_plan *p, SpinCase &c) {
  const int f = c.flip;
  const int64_t oa = c.oa, va = c.va, ob = c.ob, vb = c.vb;
  const int64_t np = npair(va);
  const int64_t ld1 = va * pad4(vb), ld2 = vb * pad4(va), ldP = pad4(np);
  const int nset = p->ft ? 2 : 1;
  int64_t offs[2][3];
  int64_t stride = 0;
  for (int x = 0; x < nset; ++x) {
    offs[x][0] = stride;
    stride += pad32(va * ld1);
    offs[x][1] = stride;
    stride += pad32(va * ld2);
    offs[x][2] = stride;
    stride += pad32(vb * ldP);
  }
  // block roles (src/pt.c:521-529): flip swaps alpha and beta
  const int Taa = f ? 2 : 0, Tab = f ? 3 : 1, Tba = f ? 1 : 3;
  for (int x = 0; x < nset; ++x) {
    const OperandSet &S = x ? p->R : p->L;
    const int m = 12 * x;
    int r;
    const int A0 = fam_a(p, x, Taa), A1 = fam_a(p, x, Tab),
              A3 = fam_a(p, x, Tba);
    const int B0 = fam_b(p, x, Taa), B1 = fam_b(p, x, Tab),
              B3 = fam_b(p, x, Tba);
    if ((r = reg_a(p, c, m + 0, S.tau[Taa], va, va, oa, oa, A0, 0))) return r;
    if ((r = reg_a(p, c, m + 1, S.tau[Tab], vb, va, ob, oa, A1, 0))) return r;
    if ((r = reg_a(p, c, m + 2, S.tau[Tba], va, vb, oa, ob, A3, 0))) return r;
    if ((r = reg_a(p, c, m + 3, S.oovo[Taa], oa, va, oa, oa, A0, 1))) return r;
    if ((r = reg_a(p, c, m + 4, S.oovo[Tab], ob, va, ob, oa, A1, 1))) return r;
    if ((r = reg_a(p, c, m + 5, S.oovo[Tba], oa, vb, oa, ob, A3, 1))) return r;
    if ((r = reg_ovvv(p, c, m + 6, S, Taa, np, ldP, va, oa, B0))) return r;
    if ((r = reg_ovvv(p, c, m + 7, S, Tab, ld1, ld1, vb, oa, B1))) return r;
    if ((r = reg_ovvv(p, c, m + 8, S, Tba, ld2, ld2, va, ob, B3))) return r;
    if ((r = reg_b(p, c, m + 9, S.taup[f], np, ldP, oa, oa, B0, 1))) return r;
    if ((r = reg_b(p, c, m + 10, S.tau[Tab], ld1, ld1, ob, oa, B1, 1))) return r;
    if ((r = reg_b(p, c, m + 11, S.tau[Tba], ld2, ld2, oa, ob, B3, 1))) return r;
    const int b = 12 * x;
    JobT u1, u2, pp;
    // U1[x][y,c] = -t_ik I_j + t_jk I_i + O_jk t_i - O_ik t_j
    u1.off = offs[x][0];
    u1.M = (int)va;
    u1.N = (int)ld1;
    u1.ldc = ld1;
    u1.nseg = 4;
    u1.seg[0] = seg(b + 1, b + 7, true, K, I, J, vb);
    u1.seg[1] = seg(b + 1, b + 7, false, K, J, I, vb);
    u1.seg[2] = seg(b + 4, b + 10, false, K, J, I, ob);
    u1.seg[3] = seg(b + 4, b + 10, true, K, I, J, ob);
    // U2[x][c,y] = -t_ij I_k + O_ji t_k
    u2.off = offs[x][1];
    u2.M = (int)va;
    u2.N = (int)ld2;
    u2.ldc = ld2;
    u2.nseg = 2;
    u2.seg[0] = seg(b + 0, b + 8, true, J, I, K, va);
    u2.seg[1] = seg(b + 3, b + 11, false, I, J, K, oa);
    // P[c][pair] = -t_kj I_i + t_ki I_j - O_kj tp_i + O_ki tp_j
    pp.off = offs[x][2];
    pp.M = (int)vb;
    pp.N = (int)ldP;
    pp.ldc = ldP;
    pp.nseg = 4;
    pp.seg[0] = seg(b + 2, b + 6, true, J, K, I, va);
    pp.seg[1] = seg(b + 2, b + 6, false, I, K, J, va);
    pp.seg[2] = seg(b + 5, b + 9, true, J, K, I, oa);
    pp.seg[3] = seg(b + 5, b + 9, false, I, K, J, oa);
    c.jobs.push_back(u1);
    c.jobs.push_back(u2);
    if (np > 0) c.jobs.push_back(pp);
  }
  EpiArgs &e = c.epi;
  memset(&e, 0, sizeof(e));
  c.ws_stride = stride;
  for (int q = 0; q < 3; ++q) {
    e.offL[q] = offs[0][q];
    e.offR[q] = p->ft ? offs[1][q] : -1;
  }
  e.ld[0] = ld1;
  e.ld[1] = ld2;
  e.ld[2] = ldP;
  e.rowU1 = pad4(vb);
  e.rowU2 = pad4(va);
  e.oa = (int)oa;
  e.va = (int)va;
  e.ob = (int)ob;
  e.vb = (int)vb;
  const int64_t offA = f ? (int64_t)p->oa * p->va : 0;
  const int64_t offB = f ? 0 : (int64_t)p->oa * p->va;
  const int64_t offB_r = p->unrestricted ? offB : 0;
  e.d_a = p->d_ov + offA;
  e.d_b = p->d_ov + offB_r;
  e.ov1_a = p->ov1 + offA;
  e.ov1_b = p->ov1 + offB_r;
  e.ov2_a = p->ov2 + offA;
  e.ov2_b = p->ov2 + offB_r;
  e.g1_ab = p->oovv[Tab];
  e.g1_ld_ab = vb;
  e.g1_aa = p->oovv[Taa];
  e.g1_ld_aa = va;
  e.g2_ab = p->L.tau[Tab];
  e.g2_ld_ab = pad4(vb);
  e.g2_aa = p->L.tau[Taa];
  e.g2_ld_aa = pad4(va);
  std::vector<int4> tiles;
  for (int64_t a0 = 0; a0 < va; a0 += EPI_A) {
    const int64_t amax = std::min<int64_t>(a0 + EPI_A - 1, va - 1);
    for (int64_t b0 = 0; b0 <= a0; b0 += EPI_B)
      if (amax - 1 >= b0) tiles.push_back(make_int4((int)a0, (int)b0, 0, 0));
  }
  c.ctiles = (int)((vb + EPI_C - 1) / EPI_C);
  c.ntiles = (int)tiles.size() * c.ctiles;
  if (!tiles.empty()) {
    if (dalloc(p, (void **)&c.d_tiles, tiles.size() * sizeof(int4))) return LIBPT_ERR_NOMEM;
    DEV(cudaMemcpyAsync(c.d_tiles, tiles.data(), tiles.size() * sizeof(int4),
                       cudaMemcpyHostToDevice, p->st));
    DEV(cudaStreamSynchronize(p->st));
  }
  e.ntiles = c.ntiles;
  e.tiles = c.d_tiles;
  e.ctiles = c.ctiles;
  e.has_f = p->has_f ? 1 : 0;
  const double A = (double)va, B = (double)vb;
  c.flops_per_triple = 2 * A * A * A * B + 4 * A * A * B * B +
                       2 * B * A * A * (A - 1) + 6 * A * A * B * oa +
                       4 * A * A * B * ob;
  if (p->ft) c.flops_per_triple *= 2;
  return LIBPT_OK;
}

Family *family(libpt_plan *p, int id, int64_t n) {
  for (Family &f : p->fams)
    if (f.id == id) return &f;
  Family f;
  f.id = id;
  f.n = n;
  if (dalloc(p, (void **)&f.max0, n * 8 + 8) ||
      dalloc(p, (void **)&f.max1, n * 8 + 8) || dalloc(p, (void **)&f.e, n + 16))
    return nullptr;
  if (!g_dry) {
    cudaMemsetAsync(f.max0, 0, n * 8 + 8, p->st);
    cudaMemsetAsync(f.max1, 0, n * 8 + 8, p->st);
  }
  p->fams.push_back(f);
  return &p->fams.back();
}

// Emulated FP64, phase 1: per-row / per-column maxima of every operand of
// every case, into its family's part (each operand once).
int i8_maxima(libpt_plan *p) {
  std::vector<std::pair<const double *, int>> seen;
  for (SpinCase &c : p->cases) {
    if (c.count == 0) continue;
    for (int i = 0; i < MAX_MAPS; ++i) {
      const OpDesc &d = c.opd[i];
      if (d.role < 0) continue;
      Family *f = family(p, d.fam, d.role == 0 ? d.R : d.N);
      if (!f) return LIBPT_ERR_NOMEM;
      const std::pair<const double *, int> key(d.src, d.role * 2 + d.part);
      if (std::find(seen.begin(), seen.end(), key) != seen.end()) continue;
      seen.push_back(key);
      unsigned long long *m = d.part ? f->max1 : f->max0;
      if (d.role == 0)
        DEV(rowmax_launch(d.src, d.P * d.Q, d.R, d.K, pad4(d.K), m, p->st));
      else
        DEV(colmax_launch(d.src, d.P, d.K, d.N, d.w, d.wsrc, d.ldsrc, m, p->st));
    }
  }
  return LIBPT_OK;
}

// Phase 2: per operand set, the power-of-two exchange between the OOVO and
// the amplitude operand sides that balances their magnitudes; phase 3: the
// joint exponents of every family.
int i8_exponents(libpt_plan *p) {
  std::vector<unsigned long long> h;
  for (int x = 0; x < (p->ft ? 2 : 1); ++x) {
    double m0 = 0.0, m1 = 0.0;
    for (Family &f : p->fams) {
      if (f.id >= 100 || f.id / 8 != x) continue;   // A families of set x
      for (int part = 0; part < 2; ++part) {
        h.assign(f.n, 0);
        DEV(cudaMemcpyAsync(h.data(), part ? f.max1 : f.max0, f.n * 8,
                            cudaMemcpyDeviceToHost, p->st));
        DEV(cudaStreamSynchronize(p->st));
        for (unsigned long long u : h) {
          double v;
          memcpy(&v, &u, 8);
          (part ? m1 : m0) = std::max(part ? m1 : m0, v);
        }
      }
    }
    OperandSet &S = x ? p->R : p->L;
    S.balance = (m0 > 0 && m1 > 0) ? (int)std::lround(std::log2(m1 / m0)) : 0;
  }
  for (Family &f : p->fams) {
    const int set = (f.id % 100) / 8;
    const int k = (set ? p->R : p->L).balance;
    const double s1 = std::ldexp(1.0, f.id >= 100 ? k : -k);
    DEV(exps_launch(f.max0, f.max1, s1, f.n, f.e, p->st));
  }
  return LIBPT_OK;
}

// Phase 4: digit planes of every operand and the INT8 tensor-core views.
// Tensor maps of a case's digit planes for the plan's current tile variant.
int i8_encode(libpt_plan *p, SpinCase &c) {
  for (int i = 0; i < MAX_MAPS; ++i) {
    const OpDesc &d = c.opd[i];
    if (d.role < 0) continue;
    const int r =
        d.role == 0
            ? i8_map_a(&c.tcmaps.m[i], c.i8pl[i], d.K, d.R, d.Q, d.P,
                       p->slices_store)
            : i8_map_b(&c.tcmaps.m[i], c.i8pl[i], d.K, d.N, d.P,
                       p->slices_store,
                       // a CTA of a pair tile loads half of its columns
                       p->i8tile.pair ? p->i8tile.bn / 2 : p->i8tile.bn);
    if (r) return r;
  }
  return LIBPT_OK;
}

// Digit planes of a case's operands (shared between cases by source).
int i8_planes(libpt_plan *p, SpinCase &c) {
  const int S = p->slices_store;
  for (int i = 0; i < MAX_MAPS; ++i) {
    const OpDesc &d = c.opd[i];
    if (d.role < 0) continue;
    Family *f = family(p, d.fam, d.role == 0 ? d.R : d.N);
    if (!f) return LIBPT_ERR_NOMEM;
    const int set = (d.fam % 100) / 8;
    const int k = (set ? p->R : p->L).balance;
    const int64_t kpi = i8_kpad(d.K);
    const std::pair<const double *, int> key(d.src, d.role);
    signed char *pl = nullptr;
    for (auto &e : p->i8planes)
      if (e.first == key) pl = e.second;
    if (!pl) {
      const int64_t n = d.role == 0 ? d.P * d.Q * d.R * kpi : d.P * d.N * kpi;
      if (dalloc(p, (void **)&pl, (d.role == 0 ? 2 : 1) * S * n))
        return LIBPT_ERR_NOMEM;
      p->i8planes.push_back({key, pl});
      if (d.role == 0)
        DEV(slice_a_launch(d.src, d.P * d.Q, d.R, d.K, pad4(d.K), kpi,
                          std::ldexp(1.0, d.part ? -k : 0), f->e, S, p->dbits,
                          pl, p->st));
      else
        DEV(slice_b_launch(d.src, d.P, (int)d.K, d.N, d.w, d.wsrc, d.ldsrc, kpi,
                          std::ldexp(1.0, d.part ? k : 0), f->e, S, p->dbits,
                          pl, p->st));
    }
    c.i8pl[i] = pl;
  }
  if (int r = i8_encode(p, c)) return r;
  // each job's output rows / columns take the scales of its operand families
  for (JobT &j : c.jobs) {
    for (Family &f : p->fams) {
      if (f.id == c.opd[j.seg[0].amap].fam) j.ea = f.e;
      if (f.id == c.opd[j.seg[0].bmap].fam) j.eb = f.e;
    }
  }
  return LIBPT_OK;
}

// Digit width of the INT8 planes.  Every accumulator (one digit-weight
// diagonal: at most S digit products per unit of K, summed over a job's
// segments) must stay below 2^31: S * 64^2 per unit of K for 7-bit digits,
// S * 128^2 for 8-bit ones.  8-bit digits (8 bits of the operand per lower
// plane instead of 7) are used for S <= 6 whenever they fit, unless
// LIBPT_EMU_DIGITS=7; a plan that chooses S itself then stores 6 planes
// (47 bits, about as accurate as 7 planes of 7 bits).
int choose_digits(libpt_plan *p) {
  int64_t kmax = 0;
  for (const SpinCase &c : p->cases)
    for (const JobT &j : c.jobs) {
      int64_t k = 0;
      for (int s = 0; s < j.nseg; ++s) k += j.seg[s].k;
      kmax = std::max(kmax, k);
    }
  const char *env = std::getenv("LIBPT_EMU_DIGITS");
  const bool allow8 = !(env && std::atoi(env) == 7);
  auto fits8 = [&](int S) {
    return allow8 && S <= 6 && (double)kmax * S * 16384.0 < 2147483648.0;
  };
  if (p->slices_auto) {
    const int S = fits8(6) ? 6 : TC_S_MAX;
    p->dbits = S == 6 ? 8 : 7;
    p->slices = p->slices_store = S;
    const I8Tile *t = nullptr;
    if (i8_tiles(S, &t) > 0) p->i8tile = t[0];
  } else {
    p->dbits = fits8(p->slices_store) ? 8 : 7;
  }
  if (p->dbits == 7 &&
      (double)kmax * 4096.0 * p->slices_store >= 2147483648.0) {
    set_error("emulated FP64: contraction too long for exact INT32 "
              "accumulation");
    return LIBPT_ERR_UNSUPPORTED;
  }
  return LIBPT_OK;
}

int add_cases(libpt_plan *p) {
  const int oa = p->oa, va = p->va, ob = p->ob, vb = p->vb;
  auto add = [&](int type, int flip, int o1, int v1, int o2, int v2) {
    SpinCase c;
    c.type = type;
    c.flip = flip;
    c.oa = o1;
    c.va = v1;
    c.ob = o2;
    c.vb = v2;
    c.first = (int64_t)p->queue.size();
    const int ci = (int)p->cases.size();
    // src/pt.c:195-196, 318-319: an empty space contributes nothing
    const bool empty = type == 0 ? (o1 == 0 || v1 == 0)
                                 : (o1 == 0 || v1 == 0 || o2 == 0 || v2 == 0);
    if (!empty) {
      if (type == 0) {
        for (int i = 0; i < o1; ++i)
          for (int j = i + 1; j < o1; ++j)
            for (int k = j + 1; k < o1; ++k)
              p->queue.push_back(make_int4(ci, i, j, k));
      } else {
        for (int i = 0; i < o1; ++i)
          for (int j = i + 1; j < o1; ++j)
            for (int k = 0; k < o2; ++k)
              p->queue.push_back(make_int4(ci, i, j, k));
      }
    }
    c.count = (int64_t)p->queue.size() - c.first;
    p->cases.push_back(c);
  };
  add(0, 0, oa, va, oa, va);
  if (p->unrestricted) add(0, 1, ob, vb, ob, vb);
  add(1, 0, oa, va, ob, vb);
  if (p->unrestricted) add(1, 1, ob, vb, oa, va);
  for (SpinCase &c : p->cases) {
    if (c.count == 0) continue;
    // CTA tile rows: the choice that pads the GEMM rows (va, and vb for the
    // mixed-spin P job) least; ties go to 128 (more CTAs)
    auto padded = [](int64_t m, int64_t bm) { return (m + bm - 1) / bm * bm; };
    const int64_t w128 = padded(c.va, 128) + (c.type ? padded(c.vb, 128) : 0);
    const int64_t w96 = padded(c.va, 96) + (c.type ? padded(c.vb, 96) : 0);
    c.bm = w96 < w128 ? 96 : 128;
    int r = c.type == 0 ? build_aaa(p, c) : build_aab(p, c);
    if (!r && p->precision == LIBPT_PREC_TF32X3) r = build_tc(p, c);
    if (r) return r;
  }
  if (p->precision == LIBPT_PREC_EMU64) {
    if (int r = choose_digits(p)) return r;
    if (int r = i8_maxima(p)) return r;
    if (int r = i8_exponents(p)) return r;
    for (SpinCase &c : p->cases)
      if (c.count)
        if (int r = i8_planes(p, c)) return r;
  }
  return LIBPT_OK;
}

// Copies each case's kernel views (tensor maps) and epilogue arguments to
// device memory, where the kernels read them.  Re-run after any map change.
int upload_views(libpt_plan *p) {
  for (SpinCase &c : p->cases) {
    if (!c.count) continue;
    const size_t mb = sizeof(TcMapSet);   // >= sizeof(MapSet)
    if (!c.d_maps && dalloc(p, (void **)&c.d_maps, mb)) return LIBPT_ERR_NOMEM;
    if (!c.d_epi && dalloc(p, (void **)&c.d_epi, sizeof(EpiArgs)))
      return LIBPT_ERR_NOMEM;
    const void *src = p->precision == LIBPT_PREC_FP64
                          ? (const void *)&c.maps
                          : (const void *)&c.tcmaps;
    const size_t n = p->precision == LIBPT_PREC_FP64 ? sizeof(MapSet)
                                                     : sizeof(TcMapSet);
    DEV(cudaMemcpyAsync(c.d_maps, src, n, cudaMemcpyHostToDevice, p->st));
    DEV(cudaMemcpyAsync(c.d_epi, &c.epi, sizeof(EpiArgs),
                       cudaMemcpyHostToDevice, p->st));
  }
  // the sources are members of the plan, copied before they can change
  DEV(cudaStreamSynchronize(p->st));
  return LIBPT_OK;
}

// Sizes the round resources for `ents` (up to the workspace budget): the
// contraction outputs of every triple, their partial energies and the
// round descriptors.
int ensure_capacity(libpt_plan *p, const std::vector<int64_t> &ents) {
  int64_t want = 0, biggest = 0;
  for (int64_t q : ents) {
    const int64_t st = p->cases[p->queue[q].x].ws_stride;
    want += st;
    biggest = std::max(biggest, st);
    if (want * 8 >= (int64_t)p->ws_budget) break;
  }
  if (p->arena) {   // fixed resources: rounds are cut to what they hold
    if (p->tri_cap >= 1 && biggest <= p->ws_cap) return LIBPT_OK;
    set_error("scratch arena workspace smaller than one triple");
    return LIBPT_ERR_NOMEM;
  }
  want = std::max(std::min<int64_t>(want, (int64_t)(p->ws_budget / 8)), biggest);
  const size_t tri = std::max<size_t>(
      1, std::min<size_t>({(size_t)4096, ents.size(),
                           (size_t)(want / std::max<int64_t>(p->ws_stride_min, 1))}));
  if (want <= p->ws_cap && tri <= p->tri_cap) return LIBPT_OK;
  CK(cudaStreamSynchronize(p->st));
  for (void **q : {(void **)&p->ws, (void **)&p->partials, (void **)&p->d_desc}) {
    if (!*q) continue;
    auto it = std::find(p->allocs.begin(), p->allocs.end(), *q);
    if (it != p->allocs.end()) p->allocs.erase(it);
    cudaFree(*q);
    *q = nullptr;
  }
  if (p->exec_ready) {
    p->exec.destroy();
    p->exec_ready = false;
  }
  p->ws_cap = p->part_cap = 0;
  p->tri_cap = 0;
  const int64_t part = (int64_t)tri * std::max(p->ntiles_max, 1);
  const size_t desc = Executor::bytes_for(tri, p->jobs_max);
  if (dalloc(p, (void **)&p->ws, want * 8) ||
      dalloc(p, (void **)&p->partials, part * 8) ||
      dalloc(p, (void **)&p->d_desc, desc))
    return LIBPT_ERR_NOMEM;
  if (int r = p->exec.init(p->st, p->d_desc, desc, false)) return r;
  p->exec_ready = true;
  p->ws_cap = want;
  p->part_cap = part;
  p->tri_cap = tri;
  return LIBPT_OK;
}

}  // namespace

GemmGroup plan_group(const libpt_plan *p, const SpinCase &c) {
  GemmGroup g;
  if (p->precision == LIBPT_PREC_EMU64) {
    g.kind = 2;
    g.bm = TC_BM;
    g.slices = p->slices;
    g.tile = p->i8tile;
  } else if (p->precision == LIBPT_PREC_TF32X3) {
    g.kind = 1;
    g.bm = TC_BM;
  } else {
    g.kind = 0;
    g.bm = c.bm;
  }
  return g;
}

int plan_append(libpt_plan *p, const int64_t *ents, size_t n, PlanCursor &cur,
                Round &r, size_t *taken) {
  *taken = 0;
  const bool tc = p->precision == LIBPT_PREC_TF32X3;
  const bool i8 = p->precision == LIBPT_PREC_EMU64;
  for (size_t t = 0; t < n; ++t) {
    const int4 q = p->queue[ents[t]];
    SpinCase &c = p->cases[q.x];
    const int64_t wend = cur.ws_end >= 0 ? cur.ws_end : p->ws_cap;
    const int64_t pend = cur.part_end >= 0 ? cur.part_end : p->part_cap;
    const size_t tend = cur.tri_end ? cur.tri_end : p->tri_cap;
    if (cur.triples >= tend || cur.ws + c.ws_stride > wend ||
        cur.part + c.ntiles > pend)
      break;   // the round is full for this plan
    const int ijk[3] = {q.y, q.z, q.w};
    double *ws = p->ws + cur.ws;
    double *partials = p->partials + cur.part;
    cur.ws += c.ws_stride;
    cur.part += c.ntiles;
    ++cur.triples;
    ++*taken;
    const GemmGroup grp = plan_group(p, c);
    std::vector<GemmJob> &jobs = r.gemm[grp];
    const CUtensorMap *hmaps = p->precision == LIBPT_PREC_FP64 ? c.maps.m
                                                               : c.tcmaps.m;
    const int map0 = r.maps[grp].add(c.d_maps, hmaps, tc ? TC_MAX_MAPS : MAX_MAPS);
    const int bn = tc ? TC_BN : i8 ? p->i8tile.bn : GEMM_BN;
    const int bmr = tc ? TC_BM : i8 ? (p->i8tile.pair ? 2 : 1) * TC_BM : c.bm;
    for (const JobT &jt : c.jobs) {
      GemmJob g;
      memset(&g, 0, sizeof(g));
      g.out = ws + jt.off;
      g.ldc = jt.ldc;
      g.M = jt.M;
      g.N = jt.N;
      g.ea = jt.ea;
      g.eb = jt.eb;
      g.maps = c.d_maps;
      g.map0 = map0;
      g.dbits = i8 ? p->dbits : 0;
      g.ntiles_n = (jt.N + bn - 1) / bn;
      g.mtiles = (jt.M + bmr - 1) / bmr;
      g.nseg = jt.nseg;
      for (int s = 0; s < jt.nseg; ++s) {
        const SegT &st = jt.seg[s];
        GemmSeg &gs = g.seg[s];
        gs.amap = (int16_t)(tc ? 2 * st.amap : st.amap);
        gs.bmap = (int16_t)(tc ? 2 * st.bmap : st.bmap);
        // INT8: a subtracted segment reads the negated digit planes, stored
        // after the slices_store digit planes
        gs.neg = (int16_t)(st.neg ? (i8 ? p->slices_store : 1) : 0);
        gs.a_q = ijk[st.aq];
        gs.a_p = ijk[st.ap];
        if (i8) {   // INT8 A views merge (Q, P) into one coordinate
          gs.a_q = gs.a_p * (int32_t)c.opd[st.amap].Q + gs.a_q;
          gs.a_p = 0;
        }
        gs.b_p = ijk[st.bp];
        gs.ksteps = tc ? (st.k + tc_kchunk_elems(TC_TF32) - 1) /
                             tc_kchunk_elems(TC_TF32)
                  : i8 ? (st.k + p->i8tile.kc - 1) / p->i8tile.kc
                       : st.ksteps;
        gs.half_last = (int16_t)(i8 && st.k % p->i8tile.kc != 0 &&
                                 st.k % p->i8tile.kc <= 32);
      }
      jobs.push_back(g);
    }
    EpiItem e;
    memset(&e, 0, sizeof(e));
    e.args = c.d_epi;
    e.ws = ws;
    e.partials = partials;
    e.i = q.y;
    e.j = q.z;
    e.k = q.w;
    r.epi[c.type][p->ft ? 1 : 0].push_back(e);
    r.epi_blocks[c.type][p->ft ? 1 : 0].push_back(c.ntiles);
    if (p->has_f) r.epi_hasf[c.type][p->ft ? 1 : 0] = true;
    RedItem red;
    red.partials = e.partials;
    red.dst = p->e_slot + ents[t];
    red.n = c.ntiles;
    red.pad_ = 0;
    r.red.push_back(red);
    r.gemm_flops += c.flops_per_triple;
    ++r.triples;
  }
  return LIBPT_OK;
}

namespace {

// Runs queue entries in rounds, each filling the plan's round resources.
int run_entries(libpt_plan *p, const std::vector<int64_t> &ents) {
  if (ents.empty()) return LIBPT_OK;
  if (int r = ensure_capacity(p, ents)) return r;
  Round round;
  for (size_t b0 = 0; b0 < ents.size();) {
    round.clear();
    PlanCursor cur;
    size_t taken = 0;
    if (int r = plan_append(p, ents.data() + b0, ents.size() - b0, cur, round,
                            &taken))
      return r;
    if (taken == 0) {
      set_error("a triple does not fit the round resources");
      return LIBPT_ERR_NOMEM;
    }
    b0 += taken;
    if (int r = p->exec.run(round, p->d_err, p->timing ? &p->tm : nullptr,
                            &p->launches))
      return r;
  }
  return LIBPT_OK;
}

// Device time of one run of `ents` (of case c), in milliseconds.
int probe_ms(libpt_plan *p, SpinCase &c, const std::vector<int64_t> &ents,
             float *ms) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int r = LIBPT_OK;
  CK(cudaEventRecord(e0, p->st));
  r = run_entries(p, ents);
  if (!r) {
    CK(cudaEventRecord(e1, p->st));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return r;
}

// Re-encodes a case's DMMA A views for CTA tile rows bm.
int set_bm(SpinCase &c, int bm) {
  c.bm = bm;
  for (int i = 0; i < MAX_MAPS; ++i) {
    const OpDesc &d = c.opd[i];
    if (d.role == 0)
      if (int r = map_a(&c.maps.m[i], d.src, d.K, d.R, d.Q, d.P, bm)) return r;
  }
  return LIBPT_OK;
}

// Emulated FP64 with the slice count left to the library: the digit planes
// are built with the most slices (6 of 8 bits, or 7 of 7 bits; see
// choose_digits) and any S below runs on their first S planes, which are
// the S-digit decomposition (with 8-bit digits, but for rare carries into
// the last kept digit, which stay within the same error bound).
//
// Error model.  Digits are rounded to nearest, so the dropped digit products
// of a contraction element are zero-mean and their signs vary from element
// to element; the first-order energy error of a triple, sum (2W - V) dW / D,
// is then zero-mean, and triples (different amplitude rows) err
// independently.  The solve's error with S slices is therefore a sum of N
// independent per-triple errors: about sqrt(N) * rms(e_S - e_7) (the second-
// order term sum dW^2 / D is of relative size (dW/W)^2, below 1e-18 for
// S >= 4).  A sample of n = min(N, 16) triples spread over the queue is
// evaluated with all stored planes (e_max) and with S; the smallest S with
//     3 sqrt(N) rms_sample(e_S - e_max) * factor <= LIBPT_EMU_TOL / 2
// (default tolerance 1e-6 Eh) is kept.  LIBPT_EMU_BOUND=worst replaces the
// estimate by the cancellation-free bound (N / n) sum_sample |e_S - e_max|.
// Sampling costs about 3n triples; a solve with fewer than 40n triples
// (where that would exceed ~8 % of the solve) keeps all stored planes.
int choose_slices(libpt_plan *p) {
  const size_t N = p->queue.size();
  if (!N) return LIBPT_OK;
  const size_t n = std::min<size_t>(N, 16);
  const char *bound_env = std::getenv("LIBPT_EMU_BOUND");
  const bool worst = bound_env && std::strcmp(bound_env, "worst") == 0;
  auto apply = [&](int S) -> int {
    const I8Tile *tiles = nullptr;
    if (i8_tiles(S, &tiles) <= 0) return LIBPT_ERR_ARG;
    p->slices = S;
    p->i8tile = tiles[0];
    for (SpinCase &c : p->cases)
      if (c.count)
        if (int r = i8_encode(p, c)) return r;
    return upload_views(p);
  };
  const int smax = p->slices_store;   // 6 (8-bit digits) or 7 (7-bit)
  int chosen = smax;
  if (N >= 40 * n) {
    std::vector<int64_t> ents(n);
    for (size_t t = 0; t < n; ++t) ents[t] = (int64_t)(t * N / n);
    std::vector<double> slots(N + 1), ref(n);
    auto run_with = [&](int S, std::vector<double> &out) -> int {
      if (int r = apply(S)) return r;
      if (int r = run_entries(p, ents)) return r;
      CK(cudaMemcpyAsync(slots.data(), p->e_slot, (N + 1) * 8,
                         cudaMemcpyDeviceToHost, p->st));
      CK(cudaStreamSynchronize(p->st));
      out.resize(n);
      for (size_t t = 0; t < n; ++t) out[t] = slots[(size_t)ents[t]];
      return LIBPT_OK;
    };
    auto estimate = [&](const std::vector<double> &e) {
      double sum_abs = 0.0, sum_sq = 0.0;
      for (size_t t = 0; t < n; ++t) {
        const double d = e[t] - ref[t];
        sum_abs += std::fabs(d);
        sum_sq += d * d;
      }
      return p->factor * (worst ? sum_abs * (double)N / (double)n
                                : 3.0 * std::sqrt((double)N * sum_sq / (double)n));
    };
    if (int r = run_with(smax, ref)) return r;
    // try 5 first, then 4 (if 5 passed) or 6 (if not, and 6 < smax)
    std::vector<double> e;
    auto passes = [&](int S, bool *ok) -> int {
      if (int r = run_with(S, e)) return r;
      const double est = estimate(e);
      if (tune_verbose())
        std::fprintf(stderr, "libpt slices: S=%d error estimate %.3e Eh "
                             "(%s; target %.1e)\n", S, est,
                     worst ? "cancellation-free bound" : "3 sqrt(N) rms",
                     p->emu_tol);
      *ok = est <= 0.5 * p->emu_tol;
      return LIBPT_OK;
    };
    bool ok = false;
    if (int r = passes(5, &ok)) return r;
    if (ok) {
      chosen = 5;
      if (int r = passes(4, &ok)) return r;
      if (ok) chosen = 4;
    } else if (smax > 6) {
      if (int r = passes(6, &ok)) return r;
      if (ok) chosen = 6;
    }
  } else if (tune_verbose()) {
    std::fprintf(stderr, "libpt slices: %zu triples, too few to sample: %d\n",
                 N, smax);
  }
  if (int r = apply(chosen)) return r;
  CK(cudaMemsetAsync(p->e_slot, 0, (N + 1) * 8, p->st));
  CK(cudaStreamSynchronize(p->st));
  p->launches = 0;
  return LIBPT_OK;
}

// The autotuner: picks the kernel variants of a plan by timing them on a
// probe of its triples (each candidate run twice, the second run timed),
// and remembers the choice per (kind, sizes, precision, slices, dtype).
//   FP64 DMMA:      CTA tile rows 96 or 128, per spin case
//   emulated FP64:  the INT8 tile variants of the slice count (i8_tiles)
// The probe's energies are discarded (slots reset afterwards); choices do
// not change results, only speed (each output element is accumulated in
// the same order by every variant).
// Sum over the spin cases of the autotuner's probe work (two timed runs per
// candidate on up to four triples of each case; emulated FP64: of the case
// with the most work).
double probe_flops(const libpt_plan *p, int ntiles) {
  const bool emu = p->precision == LIBPT_PREC_EMU64;
  double probe = 0.0;
  for (const SpinCase &c : p->cases)
    probe = emu ? std::max(probe, 2.0 * ntiles *
                                      (double)std::min<int64_t>(c.count, 4) *
                                      c.flops_per_triple)
                : probe + 4.0 * (double)std::min<int64_t>(c.count, 4) *
                              c.flops_per_triple;
  return probe;
}

// Whether plan creation will run autotuning probes (which read operands).
bool tune_would_probe(libpt_plan *p) {
  if (p->queue.empty() || p->precision == LIBPT_PREC_TF32X3 || g_dry)
    return false;
  const bool emu = p->precision == LIBPT_PREC_EMU64;
  const std::string key = tune_key(p->kind, p->oa, p->va, p->ob, p->vb,
                                   p->precision, emu ? p->slices : 0, p->dtype);
  std::vector<int> choice;
  if (tune_lookup(key, &choice) || !tune_enabled()) return false;
  const I8Tile *tiles = nullptr;
  const int ntiles = emu ? i8_tiles(p->slices, &tiles) : 0;
  return probe_flops(p, ntiles) <=
         0.05 * plan_flops(p, 0, (int64_t)p->queue.size());
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

int autotune(libpt_plan *p) {
  if (p->queue.empty() || p->precision == LIBPT_PREC_TF32X3) return LIBPT_OK;
  const bool emu = p->precision == LIBPT_PREC_EMU64;
  const std::string key = tune_key(p->kind, p->oa, p->va, p->ob, p->vb,
                                   p->precision, emu ? p->slices : 0, p->dtype);
  const I8Tile *tiles = nullptr;
  const int ntiles = emu ? i8_tiles(p->slices, &tiles) : 0;
  std::vector<int> choice;
  if (tune_lookup(key, &choice)) {
    if (emu && !choice.empty() && choice[0] >= 0 && choice[0] < ntiles) {
      p->i8tile = tiles[choice[0]];
      for (SpinCase &c : p->cases)
        if (c.count)
          if (int r = i8_encode(p, c)) return r;
    } else if (!emu && choice.size() == p->cases.size()) {
      for (size_t ci = 0; ci < p->cases.size(); ++ci)
        if (p->cases[ci].count && (choice[ci] == 96 || choice[ci] == 128))
          if (int r = set_bm(p->cases[ci], choice[ci])) return r;
    }
    return upload_views(p);
  }
  if (!tune_enabled()) return LIBPT_OK;
  // probe: the first triples of the case with the most work
  auto probe_of = [&](const SpinCase &c) {
    const int64_t n = std::min<int64_t>(c.count, 4);
    std::vector<int64_t> e((size_t)n);
    for (int64_t x = 0; x < n; ++x) e[(size_t)x] = c.first + x;
    return e;
  };
  {
    // a small solve keeps the defaults: its probes (two timed runs per
    // candidate) would cost more than a better tile could save
    const double probe = probe_flops(p, ntiles);
    if (probe > 0.05 * plan_flops(p, 0, (int64_t)p->queue.size())) {
      if (tune_verbose())
        std::fprintf(stderr, "libpt autotune %s: skipped (probes %.3g flops "
                             "> 5%% of the solve)\n", key.c_str(), probe);
      return LIBPT_OK;
    }
  }
  int r = LIBPT_OK;
  if (emu) {
    size_t big = 0;
    double most = -1.0;
    for (size_t ci = 0; ci < p->cases.size(); ++ci) {
      const SpinCase &c = p->cases[ci];
      const double w = (double)c.count * c.flops_per_triple;
      if (c.count && w > most) {
        most = w;
        big = ci;
      }
    }
    const std::vector<int64_t> ents = probe_of(p->cases[big]);
    int best = 0;
    float best_ms = 0.f;
    for (int t = 0; t < ntiles && !r; ++t) {
      p->i8tile = tiles[t];
      r = i8_encode(p, p->cases[big]);
      if (!r) r = upload_views(p);
      float ms = 0.f;
      if (!r) r = probe_ms(p, p->cases[big], ents, &ms);
      if (!r) r = probe_ms(p, p->cases[big], ents, &ms);
      if (!r && tune_verbose())
        std::fprintf(stderr, "libpt autotune %s: INT8 tile %dx%d, K chunk %d B: %.3f ms\n",
                     key.c_str(), (tiles[t].pair ? 2 : 1) * TC_BM, tiles[t].bn,
                     tiles[t].kc, ms);
      if (!r && (t == 0 || ms < best_ms)) {
        best = t;
        best_ms = ms;
      }
    }
    if (r) return r;
    p->i8tile = tiles[best];
    for (SpinCase &c : p->cases)
      if (c.count)
        if ((r = i8_encode(p, c))) return r;
    if ((r = upload_views(p))) return r;
    choice.assign(1, best);
  } else {
    choice.assign(p->cases.size(), 0);
    for (size_t ci = 0; ci < p->cases.size() && !r; ++ci) {
      SpinCase &c = p->cases[ci];
      if (!c.count) continue;
      const std::vector<int64_t> ents = probe_of(c);
      const int start = c.bm;
      int best = start;
      float best_ms = 0.f;
      for (int bm : {start, start == 96 ? 128 : 96}) {
        if ((r = set_bm(c, bm))) break;
        if ((r = upload_views(p))) break;
        float ms = 0.f;
        if ((r = probe_ms(p, c, ents, &ms))) break;
        if ((r = probe_ms(p, c, ents, &ms))) break;
        if (tune_verbose())
          std::fprintf(stderr, "libpt autotune %s: case %zu, DMMA tile rows %d: %.3f ms\n",
                       key.c_str(), ci, bm, ms);
        if (bm == start || ms < best_ms) {
          best = bm;
          best_ms = ms;
        }
      }
      if (!r) r = set_bm(c, best);
      if (!r) r = upload_views(p);
      choice[ci] = best;
    }
    if (r) return r;
  }
  tune_store(key, choice);
  p->launches = 0;
  // forget the probe's energies
  CK(cudaMemsetAsync(p->e_slot, 0, (p->queue.size() + 1) * 8, p->st));
  CK(cudaStreamSynchronize(p->st));
  return LIBPT_OK;
}

}  // namespace

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
      std::vector<double> f((size_t)nov);
      if (cudaMemcpy(f.data(), p->ov2, (size_t)nov * 8,
                     cudaMemcpyDeviceToHost) != cudaSuccess) {
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

int plan_run(libpt_plan *p, const int64_t *idx, size_t n) {
  if (!p->deferred.empty())
    if (int r = flush_deferred(p)) return r;
  const int64_t total = (int64_t)p->queue.size();
  std::vector<int64_t> ents(n);
  for (size_t x = 0; x < n; ++x) {
    const int64_t q = idx ? idx[x] : (int64_t)x;
    if (q < 0 || q >= total) {
      set_error("libpt_plan_run: queue index out of range");
      return LIBPT_ERR_ARG;
    }
    ents[x] = q;
  }
  return run_entries(p, ents);
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

int plan_energy(libpt_plan *p, const int64_t *idx, size_t n, double *e,
                cudaStream_t rs) {
  const size_t total = p->queue.size();
  const cudaStream_t st = rs ? rs : p->st;
  // the energy readback buffer comes from the caller's allocation hook
  double *slots = static_cast<double *>(host_alloc((total + 1) * 8));
  if (!slots) {
    set_error("host allocation hook failed");
    return LIBPT_ERR_NOMEM;
  }
  struct Guard {
    double *q;
    ~Guard() { host_free(q); }
  } guard{slots};
  CK(cudaMemcpyAsync(slots, p->e_slot, (total + 1) * 8,
                     cudaMemcpyDeviceToHost, st));
  unsigned err = 0;
  CK(cudaMemcpyAsync(&err, p->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                     st));
  CK(cudaStreamSynchronize(st));
  if (err) {
    set_error("a device-side wait exceeded its time limit");
    return LIBPT_ERR_TIMEOUT;
  }
  double s = 0.0;
  if (int r = sum_slots(slots, total, idx, n, &s)) return r;
  *e = p->factor * s;
  return LIBPT_OK;
}

double wall_seconds() {
  timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

bool profile_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("LIBPT_PROFILE");
    return e && e[0] == '1';
  }();
  return on;
}

int sum_slots(const double *slots, size_t total, const int64_t *idx, size_t n,
              double *out) {
  // Neumaier-compensated sum in queue order
  double s = 0.0, comp = 0.0;
  const size_t m = idx ? n : total;
  for (size_t x = 0; x < m; ++x) {
    const int64_t q = idx ? idx[x] : (int64_t)x;
    if (q < 0 || (size_t)q >= total) {
      set_error("energy sum: queue index out of range");
      return LIBPT_ERR_ARG;
    }
    const double v = slots[q];
    const double t = s + v;
    comp += std::fabs(s) >= std::fabs(v) ? (s - t) + v : (v - t) + s;
    s = t;
  }
  *out = s + comp;
  return LIBPT_OK;
}

int64_t shard_entries(int64_t total, int rank, int size, int64_t *idx) {
  // src/pt.c:213: triple `it` belongs to rank it % size
  if (total < 0 || size < 1 || rank < 0 || rank >= size) return -1;
  int64_t n = 0;
  for (int64_t q = rank; q < total; q += size) {
    if (idx) idx[n] = q;
    ++n;
  }
  return n;
}

int plan_run_shard(libpt_plan *p, int rank, int size) {
  const int64_t total = (int64_t)p->queue.size();
  const int64_t n = shard_entries(total, rank, size, nullptr);
  if (n < 0) {
    set_error("libpt_plan_run_shard: rank outside [0, size)");
    return LIBPT_ERR_ARG;
  }
  // every slot this rank does not own stays zero, so that summing the ranks'
  // slot arrays leaves each triple's energy exactly as its owner computed it
  CK(cudaMemsetAsync(p->e_slot, 0, (total + 1) * 8, p->st));
  std::vector<int64_t> ents((size_t)n);
  shard_entries(total, rank, size, ents.data());
  return run_entries(p, ents);
}

}  // namespace ptb
