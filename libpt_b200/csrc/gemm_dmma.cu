// FP64 contraction kernel: signed multi-segment GEMM on DMMA tensor cores.
//
// Replaces the reference's per-triple dgemm_ calls (src/pt.c:40-160): one
// CTA computes a 128 x 128 tile of one triple's contraction output, summing
// all of that output's amplitude x integral products (up to six, each with
// its own sign) in one K loop, so the permuted contributions the reference
// adds one GEMM at a time (e.g. src/pt.c:236-290) meet in the accumulator.
//
// Pipeline: warp 8 (one elected lane) stages A and B tiles with TMA into a
// GEMM_STAGES-deep ring of shared-memory buffers guarded by mbarriers;
// warps 0-7 run mma.sync.m16n8k4.f64 on 64 x 32 warp tiles.
//
// Shared-memory layouts (no swizzle; TMA boxes are 32 bytes wide):
//   A stage [k/4][m][k%4]   -- four boxes of (4 k x 128 rows)
//   B stage [n/4][k][n%4]   -- thirty-two boxes of (4 n x 16 k)
// so the fragment loads of a half-warp read 16 consecutive doubles (no bank
// conflicts) for both operands.
#include "common.cuh"
#include "engine.h"

namespace ptb {

namespace {

constexpr int BM = GEMM_BM, BN = GEMM_BN, BK = GEMM_BK, ST = GEMM_STAGES;
constexpr int NCW = GEMM_CONSUMER_WARPS;
constexpr uint32_t STAGE_BYTES = (BM * BK + BK * BN) * sizeof(double);

__device__ __forceinline__ int find_job(const GemmJob *jobs, int njobs,
                                        int tile) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].tile_begin <= tile)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(GEMM_THREADS, 1)
    gemm_dmma_kernel(const __grid_constant__ MapSet maps,
                     const GemmJob *__restrict__ jobs, int njobs,
                     unsigned *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double *sA = reinterpret_cast<double *>(smem_raw);
  double *sB = sA + ST * BM * BK;
  uint64_t *full = reinterpret_cast<uint64_t *>(sB + ST * BK * BN);
  uint64_t *empty = full + ST;

  const int tile = blockIdx.x;
  const GemmJob &job = jobs[find_job(jobs, njobs, tile)];
  const int local = tile - job.tile_begin;
  const int m0 = (local / job.ntiles_n) * BM;
  const int n0 = (local % job.ntiles_n) * BN;
  const int nseg = job.nseg;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
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
      for (int s = 0; s < nseg && ok; ++s) {
        const GemmSeg sg = job.seg[s];
        const CUtensorMap *am = &maps.m[sg.amap];
        const CUtensorMap *bm = &maps.m[sg.bmap];
        for (int ks = 0; ks < sg.ksteps; ++ks) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, err)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
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
  const int wm = (warp >> 2) * 64;   // warp tile origin in the CTA tile
  const int wn = (warp & 3) * 32;
  const int g = lane >> 2, t = lane & 3;

  double acc[4][4][4];
#pragma unroll
  for (int f = 0; f < 4; ++f)
#pragma unroll
    for (int h = 0; h < 4; ++h)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[f][h][e] = 0.0;

  // Per-lane fragment offsets inside one stage.
  int aoff[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) aoff[f] = (wm + 16 * f + g) * 4 + t;
  int boff[4];
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const int n = wn + 8 * h + g;
    boff[h] = ((n >> 2) * BK + t) * 4 + (n & 3);
  }

  int stage = 0;
  uint32_t phase = 0;
  bool ok = true;
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
        double a0[4], a1[4], b[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          a0[f] = flip_sign(A[kq * BM * 4 + aoff[f]], mask);
          a1[f] = flip_sign(A[kq * BM * 4 + aoff[f] + 32], mask);
        }
#pragma unroll
        for (int h = 0; h < 4; ++h) b[h] = B[kq * 16 + boff[h]];
#pragma unroll
        for (int f = 0; f < 4; ++f)
#pragma unroll
          for (int h = 0; h < 4; ++h) dmma_16x8x4(acc[f][h], a0[f], a1[f], b[h]);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[stage]);
      if (++stage == ST) {
        stage = 0;
        phase ^= 1u;
      }
    }
  }
  if (!ok) return;

  // ---------------- store ----------------
  double *out = job.out;
  const int64_t ldc = job.ldc;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const int r = m0 + wm + 16 * f + g;
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int c = n0 + wn + 8 * h + 2 * t;
      if (c < job.N) {
        if (r < job.M)
          *reinterpret_cast<double2 *>(out + (int64_t)r * ldc + c) =
              make_double2(acc[f][h][0], acc[f][h][1]);
        if (r + 8 < job.M)
          *reinterpret_cast<double2 *>(out + (int64_t)(r + 8) * ldc + c) =
              make_double2(acc[f][h][2], acc[f][h][3]);
      }
    }
  }
}

}  // namespace

size_t gemm_smem_bytes() {
  return (size_t)ST * STAGE_BYTES + 2 * ST * sizeof(uint64_t);
}

cudaError_t gemm_dmma_launch(const MapSet &maps, const GemmJob *d_jobs,
                             int njobs, int total_tiles, unsigned *d_err,
                             cudaStream_t st) {
  if (total_tiles <= 0) return cudaSuccess;
  static bool configured = false;
  const size_t smem = gemm_smem_bytes();
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(
        gemm_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  gemm_dmma_kernel<<<total_tiles, GEMM_THREADS, smem, st>>>(maps, d_jobs,
                                                            njobs, d_err);
  return cudaGetLastError();
}

}  // namespace ptb
