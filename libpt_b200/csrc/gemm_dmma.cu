// FP64 contraction kernel: signed multi-segment GEMM on DMMA tensor cores.
//
// Replaces the reference's per-triple dgemm_ calls (src/pt.c:40-160): one
// CTA computes a BM x 128 tile of one triple's contraction output, summing
// all of that output's amplitude x integral products (up to six, each with
// its own sign) in one K loop, so the permuted contributions the reference
// adds one GEMM at a time (e.g. src/pt.c:236-290) meet in the accumulator.
//
// Pipeline: warp 8 (one elected lane) stages A and B tiles with TMA into a
// GEMM_STAGES-deep ring of shared-memory buffers guarded by mbarriers;
// warps 0-7 run mma.sync.m16n8k4.f64 on (BM/2) x 32 warp tiles.
// BM is 96 or 128 rows; the host picks the one that pads M less (v = 477
// fills 5 x 96 = 480 rows against 4 x 128 = 512).
//
// Shared-memory layouts (no swizzle; TMA boxes are 32 bytes wide):
//   A stage [k/4][m][k%4]   -- four boxes of (4 k x BM rows)
//   B stage [n/4][k][n%4]   -- thirty-two boxes of (4 n x 16 k)
// so the fragment loads of a half-warp read 16 consecutive doubles (no bank
// conflicts) for both operands.
//
// Persistent: GEMM_GRID CTAs take the launch's tiles one at a time from the
// tile queue of a device-memory work list (GemmList; common.cuh tq_*), so
// one launch can hold the triples of many plans, tiles of uneven length
// spread over the SMs, and a captured CUDA graph can be replayed with new
// lists.  The producer takes a tile, hands its index to the consumer warps
// through a shared-memory ring, and runs ahead into the next tile's operands
// while the consumers store the current one.  Each job carries its plan's
// tensor maps (device memory; fenced before first use).
//
// Tiles are numbered M-tile fastest inside a job and taken in order, so the
// CTAs that share one B (OVVV) tile run at the same time and the tile is
// fetched from DRAM once.
#include "common.cuh"
#include "engine.h"

namespace ptb {

namespace {

constexpr int BN = GEMM_BN, BK = GEMM_BK, ST = GEMM_STAGES;
constexpr int NCW = GEMM_CONSUMER_WARPS;

template <int BM>
constexpr uint32_t stage_bytes() {
  return (BM * BK + BK * BN) * sizeof(double);
}

// One CTA of GEMM_THREADS (9 warps) per SM.  With 9 warps one SM
// sub-partition hosts 3 of them, which bounds the kernel at 168 registers per
// thread (16K registers per sub-partition); the 128-row tile's 64 FP64
// accumulators per thread fit that without spilling.
template <int BM, bool PM>
__device__ __forceinline__ void dmma_body(const LaunchMaps *pm,
                                          const GemmJob *__restrict__ jobs,
                                          const int njobs, const int ntiles,
                                          GemmList *list, unsigned *err) {
  constexpr int MF = BM / 32;   // m16 fragments per warp (2 warp rows)
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double *sA = reinterpret_cast<double *>(smem_raw);
  double *sB = sA + ST * BM * BK;
  uint64_t *full = reinterpret_cast<uint64_t *>(sB + ST * BK * BN);
  uint64_t *empty = full + ST;
  TileRing *tq = reinterpret_cast<TileRing *>(empty + ST);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    tq_init(tq, NCW);
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == NCW) {
    // ---------------- producer ----------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int issued = 0;
      bool ok = true;
      int qslot = 0;
      uint32_t qph = 0;
      MapSource<PM> ms(pm);
      // tiles from the launch's queue; the next one is taken while the
      // current one is staged
      int tile = tq_take(list);
      while (ok) {
        if (!tq_put(tq, qslot, qph, tile < ntiles ? tile : -1, err) ||
            tile >= ntiles)
          break;
        const int next_tile = tq_take(list);
        const GemmJob &job =
            jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
        const int local = tile - job.tile_begin;
        const int m0 = (local % job.mtiles) * BM;
        const int n0 = (local / job.mtiles) * BN;
        const int nseg = job.nseg;
        for (int s = 0; s < nseg && ok; ++s) {
          const GemmSeg sg = job.seg[s];
          const CUtensorMap *am = ms.get(job, sg.amap);
          const CUtensorMap *bm = ms.get(job, sg.bmap);
          for (int ks = 0; ks < sg.ksteps; ++ks) {
            if (!mbar_wait(&empty[stage], phase ^ 1u, err)) {
              ok = false;
              break;
            }
            mbar_arrive_expect_tx(&full[stage], stage_bytes<BM>());
            double *dA = sA + stage * BM * BK;
            double *dB = sB + stage * BK * BN;
            const int k0 = ks * BK;
#pragma unroll
            for (int q = 0; q < BK / 4; ++q)
              tma_load_4d(dA + q * BM * 4, am, &full[stage], k0 + 4 * q, m0,
                          sg.a_q, sg.a_p);
#pragma unroll 8
            for (int r = 0; r < BN / 4; ++r)
              tma_load_3d(dB + r * BK * 4, bm, &full[stage], n0 + 4 * r, k0,
                          sg.b_p);
            ++issued;
            if (++stage == ST) {
              stage = 0;
              phase ^= 1u;
            }
          }
        }
        tile = next_tile;
      }
      tq_finish(list);
      // Drain: do not leave the CTA while copies issued by it are in flight.
      const int tail = issued < ST ? issued : ST;
      for (int d = 0; d < tail; ++d) {
        int idx = issued - 1 - d;
        mbar_wait(&full[idx % ST], (uint32_t)((idx / ST) & 1), err);
      }
    }
    return;
  }

  // ---------------- consumers ----------------
  const int wm = (warp >> 2) * (BM / 2);   // warp tile origin in the CTA tile
  const int wn = (warp & 3) * 32;
  const int g = lane >> 2, t = lane & 3;

  // Per-lane fragment offsets inside one stage.
  int aoff[MF];
#pragma unroll
  for (int f = 0; f < MF; ++f) aoff[f] = (wm + 16 * f + g) * 4 + t;
  int boff[4];
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const int n = wn + 8 * h + g;
    boff[h] = ((n >> 2) * BK + t) * 4 + (n & 3);
  }

  int stage = 0;
  uint32_t phase = 0;
  bool ok = true;
  int qslot = 0;
  uint32_t qph = 0;
  for (;;) {
    const int tile = tq_get(tq, qslot, qph, err, true);
    if (tile < 0) break;
    const GemmJob &job =
        jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
    const int local = tile - job.tile_begin;
    const int m0 = (local % job.mtiles) * BM;
    const int n0 = (local / job.mtiles) * BN;
    const int nseg = job.nseg;

    double acc[MF][4][4];
#pragma unroll
    for (int f = 0; f < MF; ++f)
#pragma unroll
      for (int h = 0; h < 4; ++h)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[f][h][e] = 0.0;

    for (int s = 0; s < nseg && ok; ++s) {
      const unsigned long long mask =
          job.seg[s].neg ? 0x8000000000000000ull : 0ull;
      const int nk = job.seg[s].ksteps;
      for (int ks = 0; ks < nk; ++ks) {
        if (!mbar_wait(&full[stage], phase, err)) {
          ok = false;
          break;
        }
        const double *A = sA + stage * BM * BK;
        const double *B = sB + stage * BK * BN;
#pragma unroll
        for (int kq = 0; kq < BK / 4; ++kq) {
          double a0[MF], a1[MF], b[4];
#pragma unroll
          for (int f = 0; f < MF; ++f) {
            a0[f] = flip_sign(A[kq * BM * 4 + aoff[f]], mask);
            a1[f] = flip_sign(A[kq * BM * 4 + aoff[f] + 32], mask);
          }
#pragma unroll
          for (int h = 0; h < 4; ++h) b[h] = B[kq * 16 + boff[h]];
#pragma unroll
          for (int f = 0; f < MF; ++f)
#pragma unroll
            for (int h = 0; h < 4; ++h)
              dmma_16x8x4(acc[f][h], a0[f], a1[f], b[h]);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stage]);
        if (++stage == ST) {
          stage = 0;
          phase ^= 1u;
        }
      }
    }
    if (!ok) break;

    // ---------------- store ----------------
    double *const out = job.out;
    const int64_t ldc = job.ldc;
    const int M = job.M, N = job.N;
#pragma unroll
    for (int f = 0; f < MF; ++f) {
      const int r = m0 + wm + 16 * f + g;
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const int c = n0 + wn + 8 * h + 2 * t;
        if (c < N) {
          if (r < M)
            *reinterpret_cast<double2 *>(out + (int64_t)r * ldc + c) =
                make_double2(acc[f][h][0], acc[f][h][1]);
          if (r + 8 < M)
            *reinterpret_cast<double2 *>(out + (int64_t)(r + 8) * ldc + c) =
                make_double2(acc[f][h][2], acc[f][h][3]);
        }
      }
    }
  }
}

template <int BM>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
    gemm_dmma_kernel(const __grid_constant__ LaunchMaps pm,
                     const GemmJob *__restrict__ jobs, int njobs, int ntiles,
                     GemmList *list, unsigned *err) {
  dmma_body<BM, true>(&pm, jobs, njobs, ntiles, list, err);
}

template <int BM>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
    gemm_dmma_kernel_dm(const GemmJob *__restrict__ jobs, GemmList *list,
                        unsigned *err) {
  dmma_body<BM, false>(nullptr, jobs, list->njobs, list->ntiles, list, err);
}

template <int BM>
cudaError_t launch(const GemmJob *d_jobs, GemmList *d_list, int njobs,
                   int ntiles, const LaunchMaps *pm, int grid, unsigned *d_err,
                   cudaStream_t st) {
  static bool configured = false;
  const size_t smem = gemm_smem_bytes(BM);
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(
        gemm_dmma_kernel<BM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(gemm_dmma_kernel_dm<BM>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  if (pm)
    gemm_dmma_kernel<BM><<<grid, GEMM_THREADS, smem, st>>>(*pm, d_jobs, njobs,
                                                           ntiles, d_list,
                                                           d_err);
  else
    gemm_dmma_kernel_dm<BM><<<grid, GEMM_THREADS, smem, st>>>(d_jobs, d_list,
                                                              d_err);
  return cudaGetLastError();
}

}  // namespace

size_t gemm_smem_bytes(int bm) {
  return (size_t)ST * (bm * BK + BK * BN) * sizeof(double) +
         2 * ST * sizeof(uint64_t) + sizeof(TileRing);
}

cudaError_t gemm_dmma_launch(const GemmJob *d_jobs, GemmList *d_list,
                             int njobs, int ntiles, const LaunchMaps *pm,
                             int bm, int grid, unsigned *d_err,
                             cudaStream_t st) {
  if (grid <= 0) return cudaSuccess;
  if (bm == 96)
    return launch<96>(d_jobs, d_list, njobs, ntiles, pm, grid, d_err, st);
  return launch<128>(d_jobs, d_list, njobs, ntiles, pm, grid, d_err, st);
}

}  // namespace ptb
