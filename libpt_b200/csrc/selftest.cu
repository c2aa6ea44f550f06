// Built-in self-test of the contraction kernels (libpt_selftest): one job
// C = A B1 - A B2 with two signed segments on random operands, compared with
// a plain FP64 product computed on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "common.cuh"
#include "plan.h"
#include "pt.h"

#define LIBPT_API extern "C" __attribute__((visibility("default")))

namespace {

// Values exactly representable in FP32 (so the TF32 planes split them
// exactly), uniform in (-1, 1), from an integer hash of (seed, index).
__global__ void fill_kernel(double *x, int64_t rows, int64_t w, int64_t ld,
                            uint32_t seed, int full) {
  const int64_t n = rows * ld;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i % ld;
    uint32_t h = (uint32_t)i * 2654435761u ^ (seed * 40503u + 0x9e3779b9u);
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    const float u = (float)(h >> 8) * (1.0f / 8388608.0f) - 1.0f;
    // full: add 29 more random bits below the FP32 value (FP64 operands)
    const double lo = full ? (double)(h & 0xFFu) * 0x1p-32 +
                                 (double)((i * 0x9E3779B97F4A7C15ull) >> 43) * 0x1p-53
                           : 0.0;
    x[i] = c < w ? (double)u + lo : 0.0;
  }
}

// C = A (B1 - B2) and its magnitude sum |A| (|B1| + |B2|), the scale that
// bounds a dot product's rounding error.
__global__ void ref_kernel(const double *A, const double *B1, const double *B2,
                           double *C, double *Cabs, int m, int n, int k,
                           int64_t lda, int64_t ldb) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)m * n) return;
  const int r = (int)(idx / n), c = (int)(idx % n);
  double s = 0.0, t = 0.0;
  for (int x = 0; x < k; ++x) {
    const double a = A[r * lda + x], b1 = B1[x * ldb + c], b2 = B2[x * ldb + c];
    s += a * (b1 - b2);
    t += fabs(a) * (fabs(b1) + fabs(b2));
  }
  C[r * ldb + c] = s;
  Cabs[r * ldb + c] = t;
}

ptb::TcMapSet &tcmaps_scratch() {
  static ptb::TcMapSet m;
  return m;
}

}  // namespace

namespace {

// One contraction job on random operands: checked against the FP64
// reference (rel_err), then, when reps > 0, launched reps more times and
// timed with CUDA events (ms: mean device time of one launch).
int kernel_case(int precision, int m, int n, int k, int reps, double *rel_err,
                double *ms) {
  using namespace ptb;
  int slices = (precision >> 8) & 0x7F;
  const int dbits = (precision >> 15) & 1 ? 8 : 7;   // digit width
  const int variant = (precision >> 16) & 0xFF;
  const bool dev_maps = ((precision >> 24) & 0xFF) != 0;
  precision &= 0xFF;
  if (slices == 0) slices = 6;
  const I8Tile *tiles = nullptr;
  const int ntiles = i8_tiles(slices, &tiles);
  const int nvar = precision == LIBPT_PREC_FP64    ? 2
                   : precision == LIBPT_PREC_EMU64 ? ntiles
                                                   : 1;
  if (!rel_err || m < 1 || n < 1 || k < 1 || m > 4096 || n > (1 << 20) ||
      k > 4096 || (int64_t)n * k > ((int64_t)1 << 27) ||
      (int64_t)m * n > ((int64_t)1 << 25) || reps < 0 ||
      slices < TC_S_MIN || slices > TC_S_MAX || (dbits == 8 && slices > 6) ||
      // 8-bit digits: the two segments' 2k products per diagonal stay
      // below 2^31 (see choose_digits in plan.cu)
      (dbits == 8 && 2.0 * k * slices * 16384.0 >= 2147483648.0) ||
      (precision != LIBPT_PREC_FP64 && precision != LIBPT_PREC_TF32X3 &&
       precision != LIBPT_PREC_EMU64) || variant >= nvar) {
    set_error("libpt_selftest: bad arguments");
    return LIBPT_ERR_ARG;
  }
  const int64_t kp = (k + 3) & ~3, np = (n + 3) & ~3;
  std::vector<void *> bufs;
  auto alloc = [&](size_t bytes) -> void * {
    void *q = nullptr;
    if (cudaMalloc(&q, bytes) != cudaSuccess) return nullptr;
    bufs.push_back(q);
    return q;
  };
  auto done = [&](int r) {
    for (void *q : bufs) cudaFree(q);
    return r;
  };
  double *A = (double *)alloc((size_t)m * kp * 8);
  double *B1 = (double *)alloc((size_t)k * np * 8);
  double *B2 = (double *)alloc((size_t)k * np * 8);
  double *Cm = (double *)alloc((size_t)m * np * 8);
  double *Cr = (double *)alloc((size_t)m * np * 8);
  double *Ca = (double *)alloc((size_t)m * np * 8);
  unsigned *err = (unsigned *)alloc(4);
  GemmJob *dj = (GemmJob *)alloc(sizeof(GemmJob));
  GemmList *dl = (GemmList *)alloc(sizeof(GemmList));
  CUtensorMap *dmaps = (CUtensorMap *)alloc(sizeof(TcMapSet));
  if (!A || !B1 || !B2 || !Cm || !Cr || !Ca || !err || !dj || !dl || !dmaps) {
    set_error("libpt_selftest: cudaMalloc failed");
    return done(LIBPT_ERR_NOMEM);
  }
  const int full = precision == LIBPT_PREC_EMU64;
  fill_kernel<<<256, 256>>>(A, m, k, kp, 1, full);
  fill_kernel<<<256, 256>>>(B1, k, n, np, 2, full);
  fill_kernel<<<256, 256>>>(B2, k, n, np, 3, full);
  cudaMemset(Cm, 0, (size_t)m * np * 8);
  cudaMemset(err, 0, 4);
  ref_kernel<<<(unsigned)(((int64_t)m * n + 255) / 256), 256>>>(
      A, B1, B2, Cr, Ca, m, n, k, kp, np);
  GemmJob job;
  memset(&job, 0, sizeof(job));
  job.out = Cm;
  job.ldc = np;
  job.M = m;
  job.N = (int)np;
  job.nseg = 2;
  int r = LIBPT_OK;
  cudaError_t ce = cudaSuccess;
  std::function<cudaError_t()> launch;
  int grid = 0, nt = 0;
  // the job, its one-entry work list and its views, in device memory
  // views as kernel parameters (bits 24-31 of the precision word select
  // device-memory views instead)
  LaunchMaps pm_host;
  const LaunchMaps *pmaps = dev_maps ? nullptr : &pm_host;
  auto publish = [&](const void *maps, size_t bytes) {
    job.maps = dmaps;
    job.map0 = 0;
    job.tile_begin = 0;
    std::memcpy(&pm_host, maps, bytes < sizeof(pm_host) ? bytes : sizeof(pm_host));
    GemmList l{};
    l.jobs = dj;
    l.njobs = 1;
    l.ntiles = job.mtiles * job.ntiles_n;
    nt = l.ntiles;
    grid = l.ntiles < GEMM_GRID ? l.ntiles : GEMM_GRID;
    cudaMemcpy(dmaps, maps, bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dj, &job, sizeof(job), cudaMemcpyHostToDevice);
    cudaMemcpy(dl, &l, sizeof(l), cudaMemcpyHostToDevice);
  };
  if (precision == LIBPT_PREC_FP64) {
    MapSet maps;
    memset(&maps, 0, sizeof(maps));
    const int bm = variant ? 96 : 128;
    if ((r = dmma_map_a(&maps.m[0], A, k, m, 1, 1, bm)) ||
        (r = dmma_map_b(&maps.m[1], B1, n, np, k, 1)) ||
        (r = dmma_map_b(&maps.m[2], B2, n, np, k, 1)))
      return done(r);
    job.mtiles = (m + bm - 1) / bm;
    job.ntiles_n = (int)((np + GEMM_BN - 1) / GEMM_BN);
    for (int s = 0; s < 2; ++s) {
      job.seg[s].amap = 0;
      job.seg[s].bmap = (int16_t)(1 + s);
      job.seg[s].neg = (int16_t)s;
      job.seg[s].ksteps = (k + GEMM_BK - 1) / GEMM_BK;
    }
    publish(&maps, sizeof(maps));
    launch = [=]() { return gemm_dmma_launch(dj, dl, 1, nt, pmaps, bm, grid, err, nullptr); };
  } else if (precision == LIBPT_PREC_EMU64) {
    // one A family (A itself) and one B family (B1 part 0, B2 part 1)
    const int S = slices;
    const int64_t kpi = i8_kpad(k);
    unsigned long long *ma = (unsigned long long *)alloc((size_t)m * 8 + 8);
    unsigned long long *mb0 = (unsigned long long *)alloc((size_t)np * 8 + 8);
    unsigned long long *mb1 = (unsigned long long *)alloc((size_t)np * 8 + 8);
    signed char *ea = (signed char *)alloc((size_t)m + 16);
    signed char *eb = (signed char *)alloc((size_t)np + 16);
    signed char *pa = (signed char *)alloc((size_t)2 * S * m * kpi);
    signed char *pb1 = (signed char *)alloc((size_t)S * np * kpi);
    signed char *pb2 = (signed char *)alloc((size_t)S * np * kpi);
    if (!ma || !mb0 || !mb1 || !ea || !eb || !pa || !pb1 || !pb2) {
      set_error("libpt_selftest: cudaMalloc failed");
      return done(LIBPT_ERR_NOMEM);
    }
    cudaMemset(ma, 0, (size_t)m * 8 + 8);
    cudaMemset(mb0, 0, (size_t)np * 8 + 8);
    cudaMemset(mb1, 0, (size_t)np * 8 + 8);
    if ((ce = rowmax_launch(A, 1, m, k, kp, ma, nullptr)) ||
        (ce = colmax_launch(B1, 1, k, np, np, np, np, mb0, nullptr)) ||
        (ce = colmax_launch(B2, 1, k, np, np, np, np, mb1, nullptr)) ||
        (ce = exps_launch(ma, nullptr, 1.0, m, ea, nullptr)) ||
        (ce = exps_launch(mb0, mb1, 1.0, np, eb, nullptr)) ||
        (ce = slice_a_launch(A, 1, m, k, kp, kpi, 1.0, ea, S, dbits, pa,
                             nullptr)) ||
        (ce = slice_b_launch(B1, 1, k, np, np, np, np, kpi, 1.0, eb, S, dbits,
                             pb1,
                             nullptr)) ||
        (ce = slice_b_launch(B2, 1, k, np, np, np, np, kpi, 1.0, eb, S, dbits,
                             pb2,
                             nullptr))) {
      set_error(cudaGetErrorString(ce));
      return done(LIBPT_ERR_CUDA);
    }
    const I8Tile tl = tiles[variant];
    if ((r = i8_map_a(&(tcmaps_scratch().m[0]), pa, k, m, 1, 1, S)) ||
        (r = i8_map_b(&(tcmaps_scratch().m[1]), pb1, k, np, 1, S,
                      tl.pair ? tl.bn / 2 : tl.bn)) ||
        (r = i8_map_b(&(tcmaps_scratch().m[2]), pb2, k, np, 1, S,
                      tl.pair ? tl.bn / 2 : tl.bn)))
      return done(r);
    const int bmr = (tl.pair ? 2 : 1) * TC_BM;
    job.mtiles = (m + bmr - 1) / bmr;
    job.ntiles_n = (int)((np + tl.bn - 1) / tl.bn);
    job.ea = ea;
    job.eb = eb;
    job.dbits = dbits;
    const int kc = tl.kc;
    for (int s2 = 0; s2 < 2; ++s2) {
      job.seg[s2].amap = 0;
      job.seg[s2].bmap = (int16_t)(1 + s2);
      job.seg[s2].neg = (int16_t)(s2 ? S : 0);   // negated planes from S on
      job.seg[s2].ksteps = (k + kc - 1) / kc;
      job.seg[s2].half_last = (int16_t)(k % kc != 0 && k % kc <= 32);
    }
    publish(&tcmaps_scratch(), sizeof(TcMapSet));
    launch = [=]() {
      return gemm_i8_launch(S, tl, dj, dl, 1, nt, pmaps, grid, err, nullptr);
    };
  } else {
    float *pl[6];
    for (int x = 0; x < 6; ++x) {
      pl[x] = (float *)alloc((size_t)(x < 2 ? m : n) * kp * 4);
      if (!pl[x]) {
        set_error("libpt_selftest: cudaMalloc failed");
        return done(LIBPT_ERR_NOMEM);
      }
    }
    if ((ce = split_tf32_launch(A, pl[0], pl[1], (int64_t)m * kp, nullptr)) ||
        (ce = transpose_split_tf32_launch(B1, pl[2], pl[3], 1, k, n, np, kp,
                                          nullptr)) ||
        (ce = transpose_split_tf32_launch(B2, pl[4], pl[5], 1, k, n, np, kp,
                                          nullptr))) {
      set_error(cudaGetErrorString(ce));
      return done(LIBPT_ERR_CUDA);
    }
    TcMapSet maps;
    memset(&maps, 0, sizeof(maps));
    for (int x = 0; x < 6; ++x) {
      r = x < 2 ? tc_map_a(&maps.m[x], pl[x], k, m, 1, 1)
                : tc_map_b(&maps.m[x], pl[x], k, n, 1);
      if (r) return done(r);
    }
    job.mtiles = (m + TC_BM - 1) / TC_BM;
    job.ntiles_n = (int)((np + TC_BN - 1) / TC_BN);
    const int kc = tc_kchunk_elems(TC_TF32);
    for (int s = 0; s < 2; ++s) {
      job.seg[s].amap = 0;
      job.seg[s].bmap = (int16_t)(2 + 2 * s);
      job.seg[s].neg = (int16_t)s;
      job.seg[s].ksteps = (k + kc - 1) / kc;
    }
    TcProducts pr;
    memset(&pr, 0, sizeof(pr));
    const int8_t pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};
    for (int q = 0; q < 3; ++q) {
      pr.pa[q] = pa[q];
      pr.pb[q] = pb[q];
    }
    pr.n = 3;
    publish(&maps, sizeof(maps));
    launch = [=]() { return gemm_tc_launch(dj, dl, 1, nt, pmaps, grid, pr, err, nullptr); };
  }
  if (ce == cudaSuccess) ce = launch();
  if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
  if (ce != cudaSuccess) {
    set_error(std::string("libpt_selftest: ") + cudaGetErrorString(ce));
    return done(LIBPT_ERR_CUDA);
  }
  unsigned herr = 0;
  cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
  std::vector<double> hm((size_t)m * np), hr((size_t)m * np),
      ha((size_t)m * np);
  cudaMemcpy(hm.data(), Cm, hm.size() * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(hr.data(), Cr, hr.size() * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(ha.data(), Ca, ha.size() * 8, cudaMemcpyDeviceToHost);
  double dmax = 0.0, rmax = 0.0;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) {
      const size_t x = (size_t)i * np + j;
      dmax = std::max(dmax, std::fabs(hm[x] - hr[x]));
      rmax = std::max(rmax, ha[x]);
    }
  *rel_err = rmax > 0 ? dmax / rmax : dmax;
  if (herr) {
    set_error("libpt_selftest: a device-side wait exceeded its time limit");
    return done(LIBPT_ERR_TIMEOUT);
  }
  if (reps > 0 && ms) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, nullptr);
    for (int x = 0; x < reps && ce == cudaSuccess; ++x) ce = launch();
    cudaEventRecord(e1, nullptr);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float t = 0.f;
    if (ce == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ce != cudaSuccess) {
      set_error(std::string("libpt_kernel_bench: ") + cudaGetErrorString(ce));
      return done(LIBPT_ERR_CUDA);
    }
    *ms = t / reps;
    cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
    if (herr) {
      set_error("libpt_kernel_bench: a device-side wait exceeded its limit");
      return done(LIBPT_ERR_TIMEOUT);
    }
    // the launches reuse one work list, whose tile queue each launch must
    // leave reset for the next: one more launch into a cleared output has
    // to reproduce the first launch's result bit for bit (each element is
    // accumulated in a fixed order by whichever CTA takes its tile)
    cudaMemset(Cm, 0, (size_t)m * np * 8);
    ce = launch();
    if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
    std::vector<double> h2((size_t)m * np);
    if (ce == cudaSuccess)
      ce = cudaMemcpy(h2.data(), Cm, h2.size() * 8, cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) {
      set_error(std::string("libpt_kernel_bench: ") + cudaGetErrorString(ce));
      return done(LIBPT_ERR_CUDA);
    }
    if (std::memcmp(h2.data(), hm.data(), h2.size() * 8) != 0) {
      set_error("libpt_kernel_bench: a relaunch of the same work list gave a "
                "different result");
      return done(LIBPT_ERR_CUDA);
    }
  }
  return done(LIBPT_OK);
}

}  // namespace

LIBPT_API int libpt_selftest(int precision, int m, int n, int k,
                             double *rel_err) {
  if (n > 4096) {
    ptb::set_error("libpt_selftest: n > 4096");
    return LIBPT_ERR_ARG;
  }
  return kernel_case(precision, m, n, k, 0, rel_err, nullptr);
}

LIBPT_API int libpt_kernel_bench(int precision, int m, int n, int k, int reps,
                                 double *ms, double *rel_err) {
  if (!ms || reps < 1) {
    ptb::set_error("libpt_kernel_bench: bad arguments");
    return LIBPT_ERR_ARG;
  }
  double e = 0.0;
  const int r = kernel_case(precision, m, n, k, reps, &e, ms);
  if (rel_err) *rel_err = e;
  return r;
}

LIBPT_API int libpt_selftest_variants(int precision) {
  int slices = (precision >> 8) & 0x7F;
  if (slices == 0) slices = 6;
  switch (precision & 0xFF) {
    case LIBPT_PREC_FP64: return 2;
    case LIBPT_PREC_TF32X3: return 1;
    case LIBPT_PREC_EMU64: {
      const ptb::I8Tile *t = nullptr;
      return ptb::i8_tiles(slices, &t);
    }
    default: return 0;
  }
}

namespace {

// Wait probe: a producer / consumer hand-off through a ring of four stages
// (the pipelines of the contraction kernels in miniature), in which the
// producer stops after `arrive` of the `stages` hand-offs -- a lost arrival,
// as a TMA completion that never comes would be.  Every wait is bounded by
// limit_ns: the consumer's wait for the missing hand-off runs out, raises
// ERR_WAIT_TIMEOUT in *err and the kernel returns; nothing spins forever.
__global__ void wait_probe_kernel(int stages, int arrive,
                                  unsigned long long limit_ns, unsigned *err,
                                  int *seen) {
  __shared__ __align__(8) uint64_t full[4], empty[4];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 4; ++i) {
      ptb::mbar_init(&full[i], 1);
      ptb::mbar_init(&empty[i], 1);
    }
    ptb::mbar_fence_init();
  }
  __syncthreads();
  if (lane != 0) return;
  if (warp == 0) {          // producer
    for (int s = 0; s < stages && s < arrive; ++s) {
      const uint32_t ph = (s >> 2) & 1;
      if (!ptb::mbar_wait(&empty[s & 3], ph ^ 1, err, limit_ns)) return;
      ptb::mbar_arrive(&full[s & 3]);
    }
  } else if (warp == 1) {   // consumer
    for (int s = 0; s < stages; ++s) {
      const uint32_t ph = (s >> 2) & 1;
      if (!ptb::mbar_wait(&full[s & 3], ph, err, limit_ns)) return;
      atomicAdd(seen, 1);
      ptb::mbar_arrive(&empty[s & 3]);
    }
  }
}

}  // namespace

// Largest distance in units in the last place between recip_nr(d) and the
// IEEE division 1.0 / d over n values d = +-2^x, x evenly spaced in
// [lo_exp, hi_exp], times a mantissa that walks [1, 2).
__global__ void recip_probe_kernel(int lo_exp, int hi_exp, int n,
                                   unsigned long long *worst) {
  unsigned long long w = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const double f = n > 1 ? (double)i / (double)(n - 1) : 0.0;
    const double x = lo_exp + f * (double)(hi_exp - lo_exp);
    const double m = 1.0 + (double)((i * 2654435761u) >> 8) * 0x1p-24;
    double d = ldexp(m, (int)floor(x));
    if (i & 1) d = -d;
    const long long a = __double_as_longlong(ptb::recip_nr(d));
    const long long b = __double_as_longlong(1.0 / d);
    const unsigned long long u =
        (unsigned long long)(a > b ? a - b : b - a);   // same sign: ulps
    w = u > w ? u : w;
  }
  atomicMax(worst, w);
}

LIBPT_API int libpt_selftest_wait(int stages, int arrive, double limit_ms,
                                  int *seen) {
  if (stages < 1 || stages > 4096 || arrive < 0 || arrive > stages ||
      !(limit_ms > 0.0) || limit_ms > 2000.0 || !seen) {
    ptb::set_error("libpt_selftest_wait: bad arguments");
    return LIBPT_ERR_ARG;
  }
  unsigned *buf = nullptr;   // [0]: error word, [1]: hand-offs seen
  CK(cudaMalloc(&buf, 2 * sizeof(unsigned)));
  cudaError_t ce = cudaMemset(buf, 0, 2 * sizeof(unsigned));
  if (ce == cudaSuccess) {
    wait_probe_kernel<<<1, 64>>>(stages, arrive,
                                 (unsigned long long)(limit_ms * 1e6), buf,
                                 reinterpret_cast<int *>(buf + 1));
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
  unsigned h[2] = {0, 0};
  if (ce == cudaSuccess) ce = cudaMemcpy(h, buf, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (ce != cudaSuccess) {
    ptb::set_error(std::string("libpt_selftest_wait: ") + cudaGetErrorString(ce));
    return LIBPT_ERR_CUDA;
  }
  *seen = (int)h[1];
  if (h[0] & ptb::ERR_WAIT_TIMEOUT) {
    ptb::set_error("libpt_selftest_wait: a device-side wait exceeded its "
                   "time limit of " + std::to_string(limit_ms) + " ms");
    return LIBPT_ERR_TIMEOUT;
  }
  return LIBPT_OK;
}

LIBPT_API int libpt_selftest_recip(int lo_exp, int hi_exp, int n,
                                   double *max_ulp) {
  if (lo_exp < -1000 || hi_exp > 1000 || lo_exp > hi_exp || n < 1 ||
      n > (1 << 28) || !max_ulp) {
    ptb::set_error("libpt_selftest_recip: bad arguments");
    return LIBPT_ERR_ARG;
  }
  unsigned long long *buf = nullptr;
  CK(cudaMalloc(&buf, sizeof(*buf)));
  cudaError_t ce = cudaMemset(buf, 0, sizeof(*buf));
  if (ce == cudaSuccess) {
    recip_probe_kernel<<<148 * 4, 256>>>(lo_exp, hi_exp, n, buf);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
  unsigned long long h = 0;
  if (ce == cudaSuccess) ce = cudaMemcpy(&h, buf, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (ce != cudaSuccess) {
    ptb::set_error(std::string("libpt_selftest_recip: ") + cudaGetErrorString(ce));
    return LIBPT_ERR_CUDA;
  }
  *max_ulp = (double)h;
  return LIBPT_OK;
}
