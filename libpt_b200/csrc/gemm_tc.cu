// Tensor-core (tcgen05) contraction kernel for the multi-segment jobs, in
// 3xTF32 form (FP32-level accuracy).
//
// Same job/segment structure as gemm_dmma.cu (one triple's contraction
// output = sum of signed amplitude x integral products), but the products
// run on the 5th-generation tensor cores with accumulators in TMEM.  Each
// operand is stored as planes {hi, lo} of its FP32 values, and a tile's
// result is hi*hi + hi*lo + lo*hi accumulated in one FP32 TMEM accumulator;
// the MMA's negate bit applies a segment's sign.  (The emulated-FP64 INT8
// kernel is gemm_i8.cu.)
//
// Warp roles (persistent CTA, one per SM):
//   warp 0      TMA producer: A and B plane tiles of one K chunk per stage
//               (swizzled, K-major)
//   warp 1      TMEM owner and MMA issuer: one thread issues tcgen05.mma for
//               every product and K step; tcgen05.commit frees the stage
//   warps 2-5   epilogue: tcgen05.ld of the finished accumulators, FP64
//               store (accumulators double buffered in TMEM so the next
//               tile's MMAs overlap the drain)
// All mbarrier waits are bounded; on expiry the kernel records the error,
// stops issuing, still releases TMEM, and returns.
#include "common.cuh"
#include "engine.h"

namespace ptb {

namespace {

constexpr int BM = TC_BM;   // 128 rows (TMEM lanes)


// Shared-memory matrix descriptor of a K-major operand stored as SW-byte
// swizzled rows (8-row core groups SW*8 bytes apart), sm_100 version 1.
template <int SW>
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr) {
  constexpr uint64_t layout = SW == 128 ? 2 : SW == 64 ? 4 : 6;
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) |
         ((uint64_t)((SW * 8) >> 4) << 32) | ((uint64_t)1 << 46) |
         (layout << 61);
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

template <int KIND>
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db,
                                       uint32_t idesc, uint32_t accum) {
  static_assert(KIND == TC_TF32, "TF32 operands");
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(
          tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
      "[%0];" ::"r"(smem_u32(bar))
      : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns of TMEM.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, "
      "[%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
        "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
        "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
        "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}

// Instruction descriptor: M = 128, N = BN, K-major TF32 A and B with FP32
// accumulation.
template <int KIND, int BN>
__host__ __device__ constexpr uint32_t tc_idesc() {
  static_assert(KIND == TC_TF32, "TF32 operands, FP32 accumulation");
  return ((1u << 4) | (2u << 7) | (2u << 10)) |
         ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

constexpr int pow2_cols(int c) {
  return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512;
}

template <int KIND, int BN, int NPL, int NACC, int ST, int SW, int NBUF>
struct TcCfg {
  static constexpr int A_TILE = BM * SW;          // bytes per A plane tile
  static constexpr int B_TILE = BN * SW;          // bytes per B plane tile
  static constexpr int STAGE = NPL * (A_TILE + B_TILE);
  static constexpr int KSTEP = 32;                // bytes of K per MMA
  static constexpr int KELEM = SW / 4;            // TF32 elements per row
  static constexpr int TMEM_COLS = pow2_cols(NBUF * NACC * BN);
  static constexpr int SMEM = ST * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  static_assert(NBUF * NACC * BN <= 512, "TMEM holds 512 columns");
  static_assert(STAGE % 1024 == 0, "stage tiles keep 1 KiB alignment");
};

template <int KIND, int BN, int NPL, int NACC, int ST, int SW, int NBUF,
          bool PM>
__device__ __forceinline__ void tc_body(const LaunchMaps *pm,
                                        const GemmJob *__restrict__ jobs,
                                        const int njobs, const int ntiles,
                                        const TcProducts &prods,
                                        unsigned *err) {
  using C = TcCfg<KIND, BN, NPL, NACC, ST, SW, NBUF>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char *smem = smem_raw + ((1024 - (raw & 1023)) & 1023);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + ST * C::STAGE);
  uint64_t *empty = full + ST;
  uint64_t *accfull = empty + ST;      // [NBUF]
  uint64_t *accempty = accfull + 2;    // [NBUF]
  uint32_t *taddr_s = reinterpret_cast<uint32_t *>(accempty + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < NBUF; ++b) {
      mbar_init(&accfull[b], 1);
      mbar_init(&accempty[b], 128);
    }
    mbar_fence_init();
  }
  if (warp == 1) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::
            "r"(smem_u32(taddr_s)),
        "r"((uint32_t)C::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *taddr_s;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer ----------------
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    MapSource<PM> ms(pm);
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      const int local = tile - job.tile_begin;
      const int m0 = (local % job.mtiles) * BM;
      const int n0 = (local / job.mtiles) * BN;
      const int nseg = job.nseg;
      for (int s = 0; s < nseg && ok; ++s) {
        const GemmSeg sg = job.seg[s];

        for (int ks = 0; ks < sg.ksteps; ++ks) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, err)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[stage], C::STAGE);
          unsigned char *st_base = smem + stage * C::STAGE;
          const int k0 = ks * C::KELEM;
#pragma unroll
          for (int p = 0; p < NPL; ++p) {
            tma_load_4d(st_base + p * C::A_TILE, ms.get(job, sg.amap + p),
                        &full[stage], k0, m0, sg.a_q, sg.a_p);
            tma_load_3d(st_base + NPL * C::A_TILE + p * C::B_TILE,
                        ms.get(job, sg.bmap + p), &full[stage], k0, n0,
                        sg.b_p);
          }
          if (++stage == ST) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles && ok;
         tile += gridDim.x, ++it) {
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      const int ab = NBUF == 2 ? (it & 1) : 0;
      const uint32_t epar = NBUF == 2 ? (uint32_t)(((it >> 1) & 1) ^ 1)
                                      : (uint32_t)((it & 1) ^ 1);
      if (!mbar_wait(&accempty[ab], epar, err)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t acc0 = tmem + (uint32_t)(ab * NACC * BN);
      uint32_t started = 0;   // bit c: accumulator c has been written
      const int nseg = job.nseg;
      for (int s = 0; s < nseg && ok; ++s) {
        const GemmSeg sg = job.seg[s];
        const uint32_t neg = sg.neg ? (1u << 13) : 0u;   // negate A
        for (int ks = 0; ks < sg.ksteps; ++ks) {
          if (!mbar_wait(&full[stage], phase, err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + stage * C::STAGE);
          const uint32_t sb = sa + NPL * C::A_TILE;
          for (int q = 0; q < prods.n; ++q) {
            const int c = prods.acc[q];
            const uint64_t da = kmajor_desc<SW>(sa + prods.pa[q] * C::A_TILE);
            const uint64_t db = kmajor_desc<SW>(sb + prods.pb[q] * C::B_TILE);
#pragma unroll
            for (int kk = 0; kk < SW / C::KSTEP; ++kk) {
              // 32-byte K steps through the swizzled row (K-major layout)
              tc_mma<KIND>(acc0 + (uint32_t)(c * BN),
                           da + (uint64_t)(kk * C::KSTEP >> 4),
                           db + (uint64_t)(kk * C::KSTEP >> 4),
                           tc_idesc<KIND, BN>() | neg, (started >> c) & 1u);
              started |= 1u << c;
            }
          }
          tc_commit(&empty[stage]);   // stage reusable once these MMAs finish
          if (++stage == ST) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (ok) tc_commit(&accfull[ab]);
    }
  } else if (warp >= 2) {
    // ---------------- epilogue ----------------
    const int q = warp & 3;            // TMEM lane quarter of this warp
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      const int local = tile - job.tile_begin;
      const int m0 = (local % job.mtiles) * BM;
      const int n0 = (local / job.mtiles) * BN;
      const int ab = NBUF == 2 ? (it & 1) : 0;
      const uint32_t fpar = NBUF == 2 ? (uint32_t)((it >> 1) & 1)
                                      : (uint32_t)(it & 1);
      if (!mbar_wait(&accfull[ab], fpar, err)) break;
      tc_fence_after();
      // job fields in registers (stores and asm clobbers force reloads)
      const int row = m0 + 32 * q + lane;
      const int N = job.N;
      const bool rok = row < job.M;
      double *const orow = job.out + (int64_t)(rok ? row : 0) * job.ldc;
      const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) +
                             (uint32_t)(ab * NACC * BN);
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 32) {
        double v[32];
        uint32_t r[32];
        tmem_ld32(tbase + c0, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int x = 0; x < 32; ++x) v[x] = (double)__uint_as_float(r[x]);
        if (rok) {
#pragma unroll
          for (int x = 0; x < 32; x += 2) {
            const int col = n0 + c0 + x;
            if (col < N) {
              *reinterpret_cast<double2 *>(orow + col) =
                  make_double2(v[x], v[x + 1]);
            }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&accempty[ab]);
    }
  }
  // all roles done: release TMEM
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     tmem),
                 "r"((uint32_t)C::TMEM_COLS));
  }
}

template <int KIND, int BN, int NPL, int NACC, int ST, int SW, int NBUF>
__global__ void __launch_bounds__(192, 1)
    gemm_tc_kernel(const __grid_constant__ LaunchMaps pm,
                   const GemmJob *__restrict__ jobs, int njobs, int ntiles,
                   const __grid_constant__ TcProducts prods, unsigned *err) {
  tc_body<KIND, BN, NPL, NACC, ST, SW, NBUF, true>(&pm, jobs, njobs, ntiles,
                                                   prods, err);
}

template <int KIND, int BN, int NPL, int NACC, int ST, int SW, int NBUF>
__global__ void __launch_bounds__(192, 1)
    gemm_tc_kernel_dm(const GemmJob *__restrict__ jobs,
                      const GemmList *__restrict__ list,
                      const __grid_constant__ TcProducts prods, unsigned *err) {
  tc_body<KIND, BN, NPL, NACC, ST, SW, NBUF, false>(
      nullptr, jobs, list->njobs, list->ntiles, prods, err);
}

template <int KIND, int BN, int NPL, int NACC, int ST, int SW, int NBUF>
cudaError_t launch(const GemmJob *d_jobs, const GemmList *d_list, int njobs,
                   int ntiles, const LaunchMaps *pm, int grid,
                   const TcProducts &prods, unsigned *d_err, cudaStream_t st) {
  using C = TcCfg<KIND, BN, NPL, NACC, ST, SW, NBUF>;
  static bool configured = false;
  auto kp = gemm_tc_kernel<KIND, BN, NPL, NACC, ST, SW, NBUF>;
  auto kd = gemm_tc_kernel_dm<KIND, BN, NPL, NACC, ST, SW, NBUF>;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(
        kp, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(kd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               C::SMEM);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  if (pm)
    kp<<<grid, 192, C::SMEM, st>>>(*pm, d_jobs, njobs, ntiles, prods, d_err);
  else
    kd<<<grid, 192, C::SMEM, st>>>(d_jobs, d_list, prods, d_err);
  return cudaGetLastError();
}

}  // namespace

int tc_kchunk_elems(int kind) { return kind == TC_TF32 ? 32 : 0; }

cudaError_t gemm_tc_launch(const GemmJob *d_jobs, GemmList *d_list,
                           int njobs, int ntiles, const LaunchMaps *pm,
                           int grid, const TcProducts &prods, unsigned *d_err,
                           cudaStream_t st) {
  if (grid <= 0) return cudaSuccess;
  return launch<TC_TF32, TC_BN, 2, 1, 2, 128, 2>(d_jobs, d_list, njobs, ntiles,
                                                 pm, grid, prods, d_err, st);
}

}  // namespace ptb
