// Emulated-FP64 contraction kernel: Ozaki-style INT8 digit planes on the
// 5th-generation tensor cores (tcgen05.mma kind::i8), exact INT32
// accumulation in TMEM.
//
// Each FP64 operand is stored as S signed INT8 digit planes of base 2^b
// (b = 7 or 8, GemmJob::dbits) of the operand scaled by a power of two per
// row (A) / column (B).  A tile's result is
//     C = 2^(ea[row] + eb[col]) * g * sum_w acc_w 2^-b(w+2),
//     acc_w = sum over digit pairs p + q = w (w <= S-1) of dA_p dB_q,
// (g = 1 for b = 7; g = 4 for b = 8, whose digits carry a factor 2 each),
// each acc_w an exact INT32 sum in its own TMEM accumulator (S accumulators
// of BN columns; S * BN <= 512).  Subtracted segments read the planes of the
// negated operand (stored after the digit planes; GemmSeg::neg holds their
// first plane), so all products accumulate with +.  The kernel may use the
// first S of more stored planes.
//
// Tile variants (BN columns, KC = 32 or 64 bytes of K per pipeline stage):
// an M=128 INT8 MMA reads (128 + BN) * 32 bytes of shared memory per
// 128 * BN * 32 multiply-adds, so wider tiles relieve shared memory and L2;
// one K step per stage allows more stages in flight.  The digit planes are
// stored in 32-byte K chunks of contiguous rows, so every TMA box (32 bytes
// x 128 or BN rows) is one contiguous block: L2 serves it in whole lines
// (row-strided 32-byte boxes cost one L2 tag request per row).  The plan's
// autotuner times the variants of its slice count and keeps the fastest.
//
// Warp roles (persistent CTA, one per SM):
//   warp 0      TMA producer: the S A planes and S B planes of one K chunk
//               per stage (32-byte boxes swizzled to 32 bytes, K-major)
//   warp 1      TMEM owner and MMA issuer (one thread): S(S+1)/2 products
//               per K step; tcgen05.commit frees the stage
//   warps 2-9   epilogue: tcgen05.ld of the S accumulators, combined exactly
//               in 64-bit integers into two partial sums, one FP64 rounding,
//               an exact power-of-two scale, FP64 store.  Two warps per TMEM
//               lane quarter split the tile's 16-column chunks, so the drain
//               (during which the single-buffered accumulators hold up the
//               next tile's MMAs) takes half as long.
// All mbarrier waits are bounded; on expiry the kernel records the error,
// stops issuing, still releases TMEM, and returns.
#include "common.cuh"
#include "engine.h"

namespace ptb {

namespace {

constexpr int BM = TC_BM;   // 128 rows (TMEM lanes)


// Shared-memory descriptor of a K-major operand stored as SW-byte swizzled
// rows (8-row core groups SW*8 bytes apart), sm_100 descriptor version 1.
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

__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t da, uint64_t db,
                                       uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
      "[%0];" ::"r"(smem_u32(bar))
      : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns of TMEM.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
        "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
        "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 2^e for |e| <= 1022, built from its bit pattern (exact).
__device__ __forceinline__ double pow2i(int e) {
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// Instruction descriptor: M = 128, N = BN, K-major signed INT8 A and B,
// INT32 accumulation.
template <int BN>
__host__ __device__ constexpr uint32_t i8_idesc() {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

constexpr int pow2_cols(int c) {
  return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512;
}

template <int S, int BN, int KC>
struct I8Cfg {
  static constexpr int KS = KC / 32;                  // MMA K steps per stage
  static constexpr int A_SUB = BM * 32;               // one 32-byte K step
  static constexpr int B_SUB = (BN * 32 + 1023) / 1024 * 1024;
  static constexpr int A_TILE = KS * A_SUB;           // per plane and stage
  static constexpr int B_TILE = KS * B_SUB;
  static constexpr int STAGE = S * (A_TILE + B_TILE);
  static constexpr int TX = S * KS * (A_SUB + BN * 32);   // bytes TMA writes
  static constexpr int ST0 = (227 * 1024 - 1024 - 256) / STAGE;
  static constexpr int ST = ST0 > 8 ? 8 : ST0;                 // stages
  static constexpr int TMEM_COLS = pow2_cols(S * BN);
  static constexpr int SMEM = ST * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  static constexpr int H = (S + 1) / 2;   // accumulators in the high sum
  static_assert(S * BN <= 512, "TMEM holds 512 columns");
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "M=128 INT8 MMA N");
  static_assert(KC == 32 || KC == 64, "K chunk is one or two MMA K steps");
  static_assert(ST >= 3, "three pipeline stages at least");
  static_assert(A_TILE % 1024 == 0, "plane tiles keep 1 KiB alignment");
};

constexpr int I8_THREADS = 320;   // producer, MMA issuer, 8 epilogue warps
constexpr int I8_EPI_THREADS = 256;

template <int S, int BN, int KC, bool PM>
__device__ __forceinline__ void i8_body(const LaunchMaps *pm,
                                        const GemmJob *__restrict__ jobs,
                                        const int njobs, const int ntiles,
                                        unsigned *err) {
  using C = I8Cfg<S, BN, KC>;
  constexpr int ST = C::ST;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char *smem = smem_raw + ((1024 - (raw & 1023)) & 1023);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + ST * C::STAGE);
  uint64_t *empty = full + ST;
  uint64_t *accfull = empty + ST;
  uint64_t *accempty = accfull + 1;
  uint32_t *taddr_s = reinterpret_cast<uint32_t *>(accempty + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, I8_EPI_THREADS);
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
      // job fields are copied to registers: the asm memory clobbers and
      // global stores below would otherwise force reloads
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      const int local = tile - job.tile_begin;
      const int m0 = (local % job.mtiles) * BM;
      const int n0 = (local / job.mtiles) * BN;
      const int nseg = job.nseg;
      for (int s = 0; s < nseg && ok; ++s) {
        const GemmSeg sg = job.seg[s];
        const int aoff = sg.neg;   // first negated digit plane, or 0
        const CUtensorMap *am = ms.get(job, sg.amap);
        const CUtensorMap *bm = ms.get(job, sg.bmap);
        for (int ks = 0; ks < sg.ksteps; ++ks) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, err)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[stage], C::TX);
          unsigned char *st_base = smem + stage * C::STAGE;
#pragma unroll
          for (int p = 0; p < S; ++p) {
#pragma unroll
            for (int kk = 0; kk < C::KS; ++kk) {
              const int kc = ks * C::KS + kk;    // 32-byte K chunk
              tma_load_5d(st_base + p * C::A_TILE + kk * C::A_SUB,
                          am, &full[stage], 0, m0, kc, sg.a_q,
                          p + aoff);
              tma_load_5d(st_base + S * C::A_TILE + p * C::B_TILE +
                              kk * C::B_SUB,
                          bm, &full[stage], 0, n0, kc, sg.b_p, p);
            }
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
      if (!mbar_wait(accempty, (uint32_t)((it & 1) ^ 1), err)) {
        ok = false;
        break;
      }
      tc_fence_after();
      uint32_t started = 0;   // bit w: accumulator w has been written
      const int nseg = job.nseg;
      for (int s = 0; s < nseg && ok; ++s) {
        const int ksteps = job.seg[s].ksteps;
        for (int ks = 0; ks < ksteps; ++ks) {
          if (!mbar_wait(&full[stage], phase, err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + stage * C::STAGE);
          const uint32_t sb = sa + S * C::A_TILE;
#pragma unroll
          for (int kk = 0; kk < C::KS; ++kk) {
#pragma unroll
            for (int pa = 0; pa < S; ++pa) {
              const uint64_t da =
                  kmajor_desc<32>(sa + pa * C::A_TILE + kk * C::A_SUB);
#pragma unroll
              for (int pb = 0; pb + pa < S; ++pb) {
                const int w = pa + pb;     // digit weight 2^-b(w+2)
                const uint64_t db =
                    kmajor_desc<32>(sb + pb * C::B_TILE + kk * C::B_SUB);
                mma_i8(tmem + (uint32_t)(w * BN), da, db, i8_idesc<BN>(),
                       (started >> w) & 1u);
                started |= 1u << w;
              }
            }
          }
          tc_commit(&empty[stage]);   // stage reusable once these MMAs finish
          if (++stage == ST) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (ok) tc_commit(accfull);
    }
  } else if (warp >= 2) {
    // ---------------- epilogue ----------------
    const int q = warp & 3;            // TMEM lane quarter of this warp
    const int half = (warp - 2) >> 2;  // which 16-column chunks it takes
    int it = 0;
    constexpr int H = C::H;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      // digit base 2^b; weights of the two partial sums: hi counts units of
      // acc_{H-1}, lo units of acc_{S-1}
      const int b = job.dbits == 8 ? 8 : 7, g = b == 8 ? 2 : 0;
      const long long base = 1ll << b;
      const double w_hi = pow2i(g - b * (H + 1)), w_lo = pow2i(g - b * (S + 1));
      const int local = tile - job.tile_begin;
      const int m0 = (local % job.mtiles) * BM;
      const int n0 = (local / job.mtiles) * BN;
      const int N = job.N;
      const signed char *const eb = job.eb;
      const int row = m0 + 32 * q + lane;
      const bool rok = row < job.M;
      double *const orow = job.out + (int64_t)(rok ? row : 0) * job.ldc;
      const int erow = rok ? job.ea[row] : 0;
      if (!mbar_wait(accfull, (uint32_t)(it & 1), err)) break;
      tc_fence_after();
      const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16);
#pragma unroll 1
      for (int c0 = 16 * half; c0 < BN; c0 += 32) {
        // exact: acc_0..acc_{H-1} and acc_H..acc_{S-1} folded by Horner in
        // base 2^b into 64-bit integers; |acc| < 2^31 and each sum has at
        // most 4 terms of base 2^7 or 3 of base 2^8 (8-bit digits only for
        // S <= 6), so |sum| < 2^53 and its conversion to double is exact
        long long hi[16], lo[16];
        {
          uint32_t r[H][16];
#pragma unroll
          for (int a = 0; a < H; ++a) tmem_ld16(tbase + a * BN + c0, r[a]);
          tmem_wait_ld();
#pragma unroll
          for (int x = 0; x < 16; ++x) {
            long long h = (int)r[0][x];
#pragma unroll
            for (int a = 1; a < H; ++a) h = h * base + (int)r[a][x];
            hi[x] = h;
          }
        }
        {
          uint32_t r[S - H][16];
#pragma unroll
          for (int a = H; a < S; ++a) tmem_ld16(tbase + a * BN + c0, r[a - H]);
          tmem_wait_ld();
#pragma unroll
          for (int x = 0; x < 16; ++x) {
            long long l = (int)r[0][x];
#pragma unroll
            for (int a = H + 1; a < S; ++a) l = l * base + (int)r[a - H][x];
            lo[x] = l;
          }
        }
        if (rok && n0 + c0 < N) {
          // the chunk's 16 column exponents in one aligned 16-byte load (the
          // exponent arrays carry 16 bytes of padding past their N entries)
          const int4 ebv = *reinterpret_cast<const int4 *>(eb + n0 + c0);
          const signed char *eb16 = reinterpret_cast<const signed char *>(&ebv);
#pragma unroll
          for (int x = 0; x < 16; x += 2) {
            const int col = n0 + c0 + x;
            if (col < N) {
              // one rounding, then exact power-of-two scales
              const double v0 = fma((double)hi[x], w_hi, (double)lo[x] * w_lo) *
                                pow2i(erow + eb16[x]);
              const double v1 =
                  fma((double)hi[x + 1], w_hi, (double)lo[x + 1] * w_lo) *
                  pow2i(erow + eb16[x + 1]);
              *reinterpret_cast<double2 *>(orow + col) = make_double2(v0, v1);
            }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(accempty);
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

template <int S, int BN, int KC>
__global__ void __launch_bounds__(I8_THREADS, 1)
    gemm_i8_kernel(const __grid_constant__ LaunchMaps pm,
                   const GemmJob *__restrict__ jobs, int njobs, int ntiles,
                   unsigned *err) {
  i8_body<S, BN, KC, true>(&pm, jobs, njobs, ntiles, err);
}

template <int S, int BN, int KC>
__global__ void __launch_bounds__(I8_THREADS, 1)
    gemm_i8_kernel_dm(const GemmJob *__restrict__ jobs,
                      const GemmList *__restrict__ list, unsigned *err) {
  i8_body<S, BN, KC, false>(nullptr, jobs, list->njobs, list->ntiles, err);
}

template <int S, int BN, int KC>
cudaError_t launch(const GemmJob *d_jobs, const GemmList *d_list, int njobs,
                   int ntiles, const LaunchMaps *pm, int grid, unsigned *d_err,
                   cudaStream_t st) {
  using C = I8Cfg<S, BN, KC>;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(
        gemm_i8_kernel<S, BN, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        C::SMEM);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(gemm_i8_kernel_dm<S, BN, KC>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               C::SMEM);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  if (pm)
    gemm_i8_kernel<S, BN, KC><<<grid, I8_THREADS, C::SMEM, st>>>(
        *pm, d_jobs, njobs, ntiles, d_err);
  else
    gemm_i8_kernel_dm<S, BN, KC><<<grid, I8_THREADS, C::SMEM, st>>>(
        d_jobs, d_list, d_err);
  return cudaGetLastError();
}

// The tile variants of each slice count, widest first.
constexpr I8Tile kTiles4[] = {{128, 32}, {128, 64}, {64, 32}, {64, 64}};
constexpr I8Tile kTiles5[] = {{96, 32}, {96, 64}, {64, 32}, {64, 64}};
constexpr I8Tile kTiles6[] = {{80, 32}, {64, 32}, {64, 64}};
constexpr I8Tile kTiles7[] = {{64, 32}};

}  // namespace

int i8_tiles(int slices, const I8Tile **out) {
  switch (slices) {
    case 4: *out = kTiles4; return 4;
    case 5: *out = kTiles5; return 4;
    case 6: *out = kTiles6; return 3;
    case 7: *out = kTiles7; return 1;
    default: *out = nullptr; return 0;
  }
}

cudaError_t gemm_i8_launch(int slices, I8Tile t, const GemmJob *d_jobs,
                           const GemmList *d_list, int njobs, int ntiles,
                           const LaunchMaps *pm, int grid, unsigned *d_err,
                           cudaStream_t st) {
  if (grid <= 0) return cudaSuccess;
#define PTB_I8(S_, BN_, KC_)                                                  \
  if (slices == S_ && t.bn == BN_ && t.kc == KC_)                             \
    return launch<S_, BN_, KC_>(d_jobs, d_list, njobs, ntiles, pm, grid,     \
                                d_err, st);
  PTB_I8(4, 128, 32) PTB_I8(4, 128, 64) PTB_I8(4, 64, 32) PTB_I8(4, 64, 64)
  PTB_I8(5, 96, 32) PTB_I8(5, 96, 64) PTB_I8(5, 64, 32) PTB_I8(5, 64, 64)
  PTB_I8(6, 80, 32) PTB_I8(6, 64, 32) PTB_I8(6, 64, 64)
  PTB_I8(7, 64, 32)
#undef PTB_I8
  return cudaErrorInvalidValue;
}

}  // namespace ptb
