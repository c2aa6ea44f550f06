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
// Operand staging.  The planes are stored in 64-byte K chunks of contiguous
// rows, and a pipeline stage holds one chunk of every plane: one TMA box of
// 64 bytes x 128 (A) or BN (B) rows per plane, swizzled to 64 bytes, K-major.
// The two 32-byte MMA K steps of a stage address the two halves of the
// swizzled rows (descriptor start + 32 bytes).  A TMA unit moves box rows
// at a roughly fixed rate, so 64-byte rows carry 1.6x the bytes per clock of
// 32-byte rows (measured on B200: 26 vs 42 bytes per clock per SM); with
// 32-byte rows the box rate, not the tensor cores, set this kernel's pace.
//
// Three forms share the warp roles:
//   one CTA       128 x BN tile; A and B read from shared memory by the MMA
//   A in TMEM     the MMA thread copies each A plane of a K step into TMEM
//                 (tcgen05.cp) and the MMAs read it there, so shared memory
//                 serves A once per plane instead of once per product
//   CTA pair      256 x BN tile on two SMs (cta_group::2), each CTA loading
//                 its 128 rows of A and half of B's columns (i8_pair_body)
// The plan's autotuner times the variants of its slice count and keeps the
// fastest.
//
// Warp roles (persistent CTA, one per SM):
//   warp 0      TMA producer: the S A planes and S B planes of one K chunk
//               per stage
//   warp 1      TMEM owner and MMA issuer (one thread): S(S+1)/2 products
//               per K step (one CTA: those of one A plane with up to
//               256 / BN adjacent B planes merged into one MMA);
//               tcgen05.commit frees the stage
//   warps 2-13  epilogue: tcgen05.ld of the S accumulators, combined exactly
//               in 64-bit integers into two partial sums, one FP64 rounding,
//               an exact power-of-two scale, FP64 store.  Three warps per
//               TMEM lane quarter split the tile's 16-column chunks, so the
//               drain (during which the single-buffered accumulators hold up
//               the next tile's MMAs) is short.
// All mbarrier waits are bounded; on expiry the kernel records the error,
// stops issuing, still releases TMEM, and returns.
#include "common.cuh"
#include "engine.h"

namespace ptb {

namespace {

constexpr int BM = TC_BM;        // 128 rows (TMEM lanes)
constexpr int KB = I8_KCHUNK;    // K bytes per stage: one 64-byte chunk
constexpr int KS = KB / 32;      // MMA K steps per stage
static_assert(KB == 64, "stages are 64-byte swizzled rows");

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

// A operand in TMEM (lane = row, 8 columns of a 32-byte K step).
__device__ __forceinline__ void mma_i8_ts(uint32_t tmem, uint32_t a_tmem,
                                          uint64_t db, uint32_t idesc,
                                          uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(
          tmem),
      "r"(a_tmem), "l"(db), "r"(idesc), "r"(accum));
}

// 128 rows x 32 bytes of a K-major shared-memory matrix into TMEM: row r to
// lane r, its bytes to 8 consecutive columns (the layout of an A operand in
// TMEM).
__device__ __forceinline__ void tmem_cp_128x256b(uint32_t taddr,
                                                 uint64_t desc) {
  asm volatile("tcgen05.cp.cta_group::1.128x256b [%0], %1;" ::"r"(taddr),
               "l"(desc));
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

// Instruction descriptor: M rows (128, or 256 for a CTA pair), N = BN,
// K-major signed INT8 A and B, INT32 accumulation.
template <int M, int BN>
__host__ __device__ constexpr uint32_t i8_idesc() {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// B planes one MMA of the one-CTA form multiplies at once: N = G * BN <= 256
// (at most 4, the most any slice count's products need).
constexpr int i8_group(int bn) {
  return 256 / bn > 4 ? 4 : (256 / bn < 1 ? 1 : 256 / bn);
}

constexpr int pow2_cols(int c) {
  return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512;
}

// Shared-memory stage layout: S A planes (rows x 64 bytes), then S B planes
// (BR rows x 64 bytes each; BR = BN, or BN/2 in a CTA pair).  TS: two TMEM
// regions of S planes x 8 columns for the A operands of the last two K steps
// follow the accumulators.
template <int S, int BN, bool TS, bool PAIR>
struct I8Cfg {
  static constexpr int BR = PAIR ? BN / 2 : BN;   // B rows this CTA loads
  static constexpr int A_TILE = BM * KB;           // per plane and stage
  static constexpr int B_TILE = BR * KB;
  static constexpr int STAGE = S * (A_TILE + B_TILE);
  static constexpr int TX = (PAIR ? 2 : 1) * STAGE;   // bytes per full phase
  static constexpr int ST0 = (227 * 1024 - 1024 - 256) / STAGE;
  static constexpr int ST = ST0 > 8 ? 8 : ST0;        // stages
  static constexpr int ACOL = S * BN;   // first TMEM column of the A regions
  static constexpr int TMEM_COLS = pow2_cols(ACOL + (TS ? 16 * S : 0));
  static constexpr int SMEM = ST * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  static_assert(ACOL + (TS ? 16 * S : 0) <= 512, "TMEM holds 512 columns");
  static_assert(!(TS && PAIR), "one form at a time");
  static_assert(PAIR ? (BN % 32 == 0 && BN >= 32 && BN <= 256)
                     : (BN % 16 == 0 && BN >= 16 && BN <= 256),
                "INT8 MMA N");
  static_assert(B_TILE % 1024 == 0 && A_TILE % 1024 == 0,
                "plane tiles keep 1 KiB alignment");
  static_assert(ST >= 2, "two pipeline stages at least");
};

// Epilogue warps per TMEM lane quarter: each drains every third 16-column
// chunk of its quarter's rows, so the drain (during which the single-
// buffered accumulators hold up the next tile's MMAs) takes a third as long
// as with one warp per quarter.
constexpr int I8_EPI_GROUPS = 3;
constexpr int I8_EPI_THREADS = 4 * I8_EPI_GROUPS * 32;
constexpr int I8_THREADS = 64 + I8_EPI_THREADS;   // producer, MMA, epilogue
// (14 warps: four of them on some SM sub-partition, whose 16K registers cap
// the kernels at 128 registers per thread.)

// Drains one tile's accumulators (this CTA's 128 rows, rows from m0): the
// S INT32 sums of each element folded exactly, rounded once, scaled and
// stored.  Called by the epilogue warps after the tile's accumulators are
// complete.  `release` runs once per thread as soon as the thread's last
// TMEM loads have completed (before that chunk's stores), so the next
// tile's MMAs may start overwriting the accumulators while it stores.
template <int S, int BN, typename Release>
__device__ __forceinline__ void i8_drain(const GemmJob &job, int m0, int n0,
                                         uint32_t tmem, int warp, int lane,
                                         Release release) {
  constexpr int H = (S + 1) / 2;
  const int q = warp & 3;            // TMEM lane quarter of this warp
  const int grp = (warp - 2) >> 2;   // which 16-column chunks it takes
  // digit base 2^b; weights of the two partial sums: hi counts units of
  // acc_{H-1}, lo units of acc_{S-1}
  const int b = job.dbits == 8 ? 8 : 7, g = b == 8 ? 2 : 0;
  const long long base = 1ll << b;
  const double w_hi = pow2i(g - b * (H + 1)), w_lo = pow2i(g - b * (S + 1));
  const int N = job.N;
  const signed char *const eb = job.eb;
  const int row = m0 + 32 * q + lane;
  const bool rok = row < job.M;
  double *const orow = job.out + (int64_t)(rok ? row : 0) * job.ldc;
  const int erow = rok ? job.ea[row] : 0;
  const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16);
  constexpr int STEP = 16 * I8_EPI_GROUPS;
  // chunks a warp drains at most
  constexpr int NCH = (BN / 16 + I8_EPI_GROUPS - 1) / I8_EPI_GROUPS;
  {
    // Each chunk is drained with one TMEM wait (S <= 5: all S loads at
    // once; else the hi and lo halves, a wait each, to bound the
    // registers); the chunks' column exponents are loaded before the first
    // TMEM load (one aligned 16-byte load each: the exponent arrays carry
    // 16 bytes of padding past their N entries); a chunk's stores are
    // issued before the next chunk's loads (its registers free), and the
    // release comes right after the last chunk's loads, before its scaling
    // and stores.  The fold is exact: acc_0..acc_{H-1} and acc_H..acc_{S-1}
    // by Horner in base 2^b into 64-bit integers; |acc| < 2^31 and each sum
    // has at most 4 terms of base 2^7 or 3 of base 2^8 (8-bit digits only
    // for S <= 6), so |sum| < 2^53 and its conversion to double is exact;
    // one rounding (the fma), then exact power-of-two scales.
    int4 ebv[NCH];
#pragma unroll
    for (int i = 0; i < NCH; ++i) {
      const int c0 = 16 * grp + i * STEP;
      ebv[i] = (c0 < BN && rok && n0 + c0 < N)
                   ? *reinterpret_cast<const int4 *>(eb + n0 + c0)
                   : make_int4(0, 0, 0, 0);
    }
    // one chunk's S accumulators folded into its rounded pre-scale values:
    // all S loads and one wait, or (fewer registers) the hi and lo halves
    // with a wait each
    auto fold_one = [&](int c0, double (&vv)[16]) {
      uint32_t r[S][16];
#pragma unroll
      for (int a = 0; a < S; ++a) tmem_ld16(tbase + a * BN + c0, r[a]);
      tmem_wait_ld();
#pragma unroll
      for (int x = 0; x < 16; ++x) {
        long long h = (int)r[0][x];
#pragma unroll
        for (int a = 1; a < H; ++a) h = h * base + (int)r[a][x];
        long long l = (int)r[H][x];
#pragma unroll
        for (int a = H + 1; a < S; ++a) l = l * base + (int)r[a][x];
        vv[x] = fma((double)h, w_hi, (double)l * w_lo);
      }
    };
    auto fold_split = [&](int c0, double (&vv)[16]) {
      long long hi[16];
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
      uint32_t r[S - H][16];
#pragma unroll
      for (int a = H; a < S; ++a) tmem_ld16(tbase + a * BN + c0, r[a - H]);
      tmem_wait_ld();
#pragma unroll
      for (int x = 0; x < 16; ++x) {
        long long l = (int)r[0][x];
#pragma unroll
        for (int a = H + 1; a < S; ++a) l = l * base + (int)r[a - H][x];
        vv[x] = fma((double)hi[x], w_hi, (double)l * w_lo);
      }
    };
    // stores of one chunk: 32-byte vectors (a full sector per row) where
    // the output's alignment allows, else 16-byte pairs
    const bool v4 = ((job.ldc & 3) == 0) &&
                    ((reinterpret_cast<uintptr_t>(job.out) & 31) == 0);
    auto store = [&](int i, const double (&vv)[16]) {
      const int c0 = 16 * grp + i * STEP;
      if (!rok || n0 + c0 >= N) return;
      const signed char *eb16 = reinterpret_cast<const signed char *>(&ebv[i]);
      if (v4) {   // N % 4 == 0: a group of four columns is whole
#pragma unroll
        for (int x = 0; x < 16; x += 4) {
          const int col = n0 + c0 + x;
          if (col < N)
            asm volatile(
                "st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(orow + col),
                "d"(vv[x] * pow2i(erow + eb16[x])),
                "d"(vv[x + 1] * pow2i(erow + eb16[x + 1])),
                "d"(vv[x + 2] * pow2i(erow + eb16[x + 2])),
                "d"(vv[x + 3] * pow2i(erow + eb16[x + 3]))
                : "memory");
        }
      } else {
#pragma unroll
        for (int x = 0; x < 16; x += 2) {
          const int col = n0 + c0 + x;
          if (col < N)
            *reinterpret_cast<double2 *>(orow + col) =
                make_double2(vv[x] * pow2i(erow + eb16[x]),
                             vv[x + 1] * pow2i(erow + eb16[x + 1]));
        }
      }
    };
    // chunks of this warp (warp-uniform)
    int nch = 0;
#pragma unroll
    for (int i = 0; i < NCH; ++i)
      if (16 * grp + i * STEP < BN) nch = i + 1;
    if (nch == 0) release();
    // all chunks but the last two: fold and store in turn; the last two are
    // both folded before the release and stored after it, so that no store
    // (32 rows of scattered sectors per instruction) delays the release
    double v[16], w[16];
#pragma unroll
    for (int i = 0; i < NCH; ++i) {
      if (i >= nch) break;
      const int c0 = 16 * grp + i * STEP;
      if (i + 2 < nch) {
        if constexpr (S <= 5) fold_one(c0, v); else fold_split(c0, v);
        store(i, v);
      } else if (i + 2 == nch) {
        if constexpr (S <= 5) fold_one(c0, v); else fold_split(c0, v);
      } else {   // the last chunk
        if (i == 0) {
          if constexpr (S <= 5) fold_one(c0, v); else fold_split(c0, v);
          release();   // this thread's TMEM loads are done
          store(i, v);
        } else {
          fold_split(c0, w);
          release();
          store(i - 1, v);
          store(i, w);
        }
      }
    }
  }
}

template <int S, int BN, bool PM, bool TS>
__device__ __forceinline__ void i8_body(const LaunchMaps *pm,
                                        const GemmJob *__restrict__ jobs,
                                        const int njobs, const int ntiles,
                                        GemmList *list, unsigned *err) {
  using C = I8Cfg<S, BN, TS, false>;
  constexpr int ST = C::ST;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char *smem = smem_raw + ((1024 - (raw & 1023)) & 1023);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + ST * C::STAGE);
  uint64_t *empty = full + ST;
  uint64_t *accfull = empty + ST;
  uint64_t *accempty = accfull + 1;
  uint64_t *regbar = accempty + 1;   // TS: A region r free again (2)
  // the tile queue's ring: read by the MMA thread and the epilogue warps
  TileRing *tq = reinterpret_cast<TileRing *>(regbar + 2);
  uint32_t *taddr_s = reinterpret_cast<uint32_t *>(tq + 1);
  static_assert((2 * ST + 4) * 8 + sizeof(TileRing) + 4 <= 256,
                "barriers, tile ring and TMEM address fit their 256 bytes");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, I8_EPI_THREADS);
    mbar_init(&regbar[0], 1);
    mbar_init(&regbar[1], 1);
    tq_init(tq, 1 + I8_EPI_THREADS / 32);   // MMA thread + epilogue warps
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
            tma_load_5d(st_base + p * C::A_TILE, am, &full[stage], 0, m0, ks,
                        sg.a_q, p + aoff);
            tma_load_5d(st_base + S * C::A_TILE + p * C::B_TILE, bm,
                        &full[stage], 0, n0, ks, sg.b_p, p);
          }
          if (++stage == ST) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      tile = next_tile;
    }
    tq_finish(list);
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    int it = 0;
    int t = 0;   // TS: MMA K steps issued (region t & 1)
    int qslot = 0;
    uint32_t qph = 0;
    for (;; ++it) {
      const int tile = tq_get(tq, qslot, qph, err, false);
      if (tile < 0) break;
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      if (!mbar_wait(accempty, (uint32_t)((it & 1) ^ 1), err)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int nseg = job.nseg;
      for (int s = 0; s < nseg && ok; ++s) {
        const int ksteps = job.seg[s].ksteps;
        const bool half_last = job.seg[s].half_last != 0;
        for (int ks = 0; ks < ksteps && ok; ++ks) {
          // K steps of this stage: the zero second half of a short last
          // chunk is skipped
          const int nkk = (half_last && ks == ksteps - 1) ? 1 : KS;
          if (!mbar_wait(&full[stage], phase, err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + stage * C::STAGE);
          // descriptors of the stage's planes: the base's plus the offset
          // / 16 (the address field holds addr / 16 < 2^14 for any shared-
          // memory address, so the sum never carries out of it); a K step's
          // 32 bytes are the first or second half of the swizzled rows
          const uint64_t da0 = kmajor_desc<KB>(sa);
          const uint64_t db0 = kmajor_desc<KB>(sa + S * C::A_TILE);
          // the first product into each accumulator (pa = 0, first K step
          // of the tile) overwrites it; every later one accumulates
          const uint32_t later = (s > 0 || ks > 0) ? 1u : 0u;
#pragma unroll
          for (int kk = 0; kk < KS; ++kk) {
            if (kk >= nkk) break;
            if constexpr (TS) {
              // region t & 1 was last read by the MMAs of K step t - 2,
              // whose completion regbar[t & 1] records
              const int r = t & 1;
              if (t >= 2 &&
                  !mbar_wait(&regbar[r], (uint32_t)(((t >> 1) & 1) ^ 1), err)) {
                ok = false;
                break;
              }
              tc_fence_after();
              const uint32_t areg = tmem + (uint32_t)(C::ACOL + r * S * 8);
#pragma unroll
              for (int pa = 0; pa < S; ++pa)
                tmem_cp_128x256b(areg + (uint32_t)(pa * 8),
                                 da0 + (uint64_t)((pa * C::A_TILE + kk * 32) >> 4));
#pragma unroll
              for (int pa = 0; pa < S; ++pa) {
#pragma unroll
                for (int pb = 0; pb + pa < S; ++pb) {
                  const int w = pa + pb;
                  const uint64_t db =
                      db0 + (uint64_t)((pb * C::B_TILE + kk * 32) >> 4);
                  mma_i8_ts(tmem + (uint32_t)(w * BN),
                            areg + (uint32_t)(pa * 8), db, i8_idesc<BM, BN>(),
                            (pa > 0 || kk > 0) ? 1u : later);
                }
              }
              tc_commit(&regbar[r]);
              ++t;
            } else {
              // A_pa times B_pb .. B_pb+g-1 in one MMA of N = g * BN: the B
              // planes lie back to back in the stage (same swizzle atoms, so
              // g planes read as one tile of g * BN rows), and the
              // accumulators of weights pa + pb .. pa + pb + g - 1 are
              // adjacent TMEM columns, so column block j of the product
              // lands in acc_{pa+pb+j}.  A_pa is read once per group
              // instead of once per product (S = 5, BN = 96: 9 MMAs and 9 A
              // reads per K step instead of 15).
#pragma unroll
              for (int pa = 0; pa < S; ++pa) {
                const uint64_t da =
                    da0 + (uint64_t)((pa * C::A_TILE + kk * 32) >> 4);
#pragma unroll
                for (int pb = 0; pb + pa < S; pb += i8_group(BN)) {
                  const int w = pa + pb;     // digit weight 2^-b(w+2)
                  const int g = S - w < i8_group(BN) ? S - w : i8_group(BN);
                  const uint64_t db =
                      db0 + (uint64_t)((pb * C::B_TILE + kk * 32) >> 4);
                  const uint32_t acc = (pa > 0 || kk > 0) ? 1u : later;
                  if (g == 4)
                    mma_i8(tmem + (uint32_t)(w * BN), da, db,
                           i8_idesc<BM, 4 * BN>(), acc);
                  else if (g == 3)
                    mma_i8(tmem + (uint32_t)(w * BN), da, db,
                           i8_idesc<BM, 3 * BN>(), acc);
                  else if (g == 2)
                    mma_i8(tmem + (uint32_t)(w * BN), da, db,
                           i8_idesc<BM, 2 * BN>(), acc);
                  else
                    mma_i8(tmem + (uint32_t)(w * BN), da, db,
                           i8_idesc<BM, BN>(), acc);
                }
              }
            }
          }
          if (!ok) break;
          tc_commit(&empty[stage]);   // stage reusable once these MMAs finish
          if (++stage == ST) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!ok) break;
      tc_commit(accfull);
    }
  } else if (warp >= 2) {
    // ---------------- epilogue ----------------
    int qslot = 0;
    uint32_t qph = 0;
    for (int it = 0;; ++it) {
      const int tile = tq_get(tq, qslot, qph, err, true);
      if (tile < 0) break;
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      const int local = tile - job.tile_begin;
      if (!mbar_wait(accfull, (uint32_t)(it & 1), err)) break;
      tc_fence_after();
      i8_drain<S, BN>(job, (local % job.mtiles) * BM,
                      (local / job.mtiles) * BN, tmem, warp, lane, [&] {
                        tc_fence_before();
                        mbar_arrive(accempty);
                      });
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

// ---------------------------------------------------------------------------
// CTA-pair form: a cluster of two CTAs on two SMs computes a 256 x BN tile
// with tcgen05.mma.cta_group::2 (M = 256).  Each CTA loads its own 128 rows
// of the A planes and half (BN/2 columns) of the B planes into its own
// shared memory; the leader CTA's one MMA thread multiplies the pair's
// operands (A rows 0-127 and B columns 0..BN/2-1 from the leader, the rest
// from its peer) into both CTAs' TMEM (each holds its 128 rows x BN
// columns of the S accumulators).  Per K step a CTA reads (128 + BN/2) rows
// from L2 instead of 128 + BN.
//
// Synchronisation (all waits bounded):
//   full[s]     leader only: its producer expects both CTAs' bytes; both
//               CTAs' TMA loads complete on it (cta_group::2 loads)
//   empty[s]    each CTA's own; the leader's MMA thread commits to both
//               (one tcgen05.commit to the pair's CTA mask)
//   accfull     each CTA's own; the leader commits to both after a tile
//   accempty    leader only: one arrive per epilogue warp of both CTAs

// M = 256 MMA of the pair.
__device__ __forceinline__ void mma_i8_pair(uint32_t tmem, uint64_t da,
                                            uint64_t db, uint32_t idesc,
                                            uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accum));
}

// Arrives, once the issuing thread's earlier MMAs complete, on the mbarrier
// at this shared-memory offset in both CTAs of the pair (a tcgen05.commit
// to a CTA mask; no data moves).
__device__ __forceinline__ void tc_commit_both(const uint64_t *bar) {
  const uint16_t both = 3;
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster."
      "multicast::cluster.b64 [%0], %1;" ::"r"(smem_u32(bar)),
      "h"(both)
      : "memory");
}

template <int S, int BN, bool PM>
__device__ __forceinline__ void i8_pair_body(const LaunchMaps *pm,
                                             const GemmJob *__restrict__ jobs,
                                             const int njobs, const int ntiles,
                                             unsigned *err) {
  using C = I8Cfg<S, BN, false, true>;
  constexpr int ST = C::ST;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  // the same offset in both CTAs (equal dynamic shared memory layouts)
  unsigned char *smem = smem_raw + ((1024 - (raw & 1023)) & 1023);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + ST * C::STAGE);
  uint64_t *empty = full + ST;
  uint64_t *accfull = empty + ST;
  uint64_t *accempty = accfull + 1;
  uint32_t *taddr_s = reinterpret_cast<uint32_t *>(accempty + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();   // 0: leader
  const bool leader = rank == 0;
  const int pair0 = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, 2 * (I8_EPI_THREADS / 32));
    mbar_fence_init();
  }
  if (warp == 1) {
    asm volatile(
        "tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::
            "r"(smem_u32(taddr_s)),
        "r"((uint32_t)C::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();   // both CTAs' barriers initialised, TMEM allocated
  tc_fence_after();
  const uint32_t tmem = *taddr_s;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    MapSource<PM> ms(pm);
    for (int tile = pair0; tile < ntiles && ok; tile += npairs) {
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      const int local = tile - job.tile_begin;
      const int m0 = (local % job.mtiles) * 2 * BM + (int)rank * BM;
      const int n0 = (local / job.mtiles) * BN + (int)rank * C::BR;
      const int nseg = job.nseg;
      for (int s = 0; s < nseg && ok; ++s) {
        const GemmSeg sg = job.seg[s];
        const int aoff = sg.neg;
        const CUtensorMap *am = ms.get(job, sg.amap);
        const CUtensorMap *bm = ms.get(job, sg.bmap);
        for (int ks = 0; ks < sg.ksteps; ++ks) {
          if (!mbar_wait(&empty[stage], phase ^ 1u, err)) {
            ok = false;
            break;
          }
          if (leader) mbar_arrive_expect_tx(&full[stage], C::TX);
          const uint32_t fb = cluster_addr(&full[stage], 0);
          unsigned char *st_base = smem + stage * C::STAGE;
#pragma unroll
          for (int p = 0; p < S; ++p) {
            tma_load_5d_pair(st_base + p * C::A_TILE, am, fb, 0, m0, ks,
                             sg.a_q, p + aoff);
            tma_load_5d_pair(st_base + S * C::A_TILE + p * C::B_TILE, bm, fb,
                             0, n0, ks, sg.b_p, p);
          }
          if (++stage == ST) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
    }
  } else if (warp == 1 && lane == 0 && leader) {
    // ---------------- MMA issuer (leader CTA) ----------------
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    int it = 0;
    for (int tile = pair0; tile < ntiles && ok; tile += npairs, ++it) {
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      if (!mbar_wait(accempty, (uint32_t)((it & 1) ^ 1), err)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int nseg = job.nseg;
      for (int s = 0; s < nseg && ok; ++s) {
        const int ksteps = job.seg[s].ksteps;
        const bool half_last = job.seg[s].half_last != 0;
        for (int ks = 0; ks < ksteps; ++ks) {
          if (!mbar_wait(&full[stage], phase, err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + stage * C::STAGE);
          const uint64_t da0 = kmajor_desc<KB>(sa);   // as in i8_body
          const uint64_t db0 = kmajor_desc<KB>(sa + S * C::A_TILE);
          const uint32_t later = (s > 0 || ks > 0) ? 1u : 0u;
          const int nkk = (half_last && ks == ksteps - 1) ? 1 : KS;
#pragma unroll
          for (int kk = 0; kk < KS; ++kk) {
            if (kk >= nkk) break;
#pragma unroll
            for (int pa = 0; pa < S; ++pa) {
              const uint64_t da =
                  da0 + (uint64_t)((pa * C::A_TILE + kk * 32) >> 4);
#pragma unroll
              for (int pb = 0; pb + pa < S; ++pb) {
                const int w = pa + pb;
                const uint64_t db =
                    db0 + (uint64_t)((pb * C::B_TILE + kk * 32) >> 4);
                mma_i8_pair(tmem + (uint32_t)(w * BN), da, db,
                            i8_idesc<2 * BM, BN>(),
                            (pa > 0 || kk > 0) ? 1u : later);
              }
            }
          }
          // both CTAs' stages are free once these MMAs finish
          tc_commit_both(&empty[stage]);
          if (++stage == ST) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (ok) tc_commit_both(accfull);
    }
  } else if (warp >= 2) {
    // ---------------- epilogue (both CTAs: own 128 rows) ----------------
    int it = 0;
    const uint32_t accempty_lead = cluster_addr(accempty, 0);
    for (int tile = pair0; tile < ntiles; tile += npairs, ++it) {
      const GemmJob &job = jobs[find_entry(jobs, njobs, tile, &GemmJob::tile_begin)];
      const int local = tile - job.tile_begin;
      if (!mbar_wait(accfull, (uint32_t)(it & 1), err)) break;
      tc_fence_after();
      i8_drain<S, BN>(job, (local % job.mtiles) * 2 * BM + (int)rank * BM,
                      (local / job.mtiles) * BN, tmem, warp, lane, [&] {
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive_cluster(accempty_lead);
                      });
    }
  }
  // all roles of both CTAs done: release TMEM
  tc_fence_before();
  __syncthreads();
  cluster_sync();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(
                     tmem),
                 "r"((uint32_t)C::TMEM_COLS));
  }
}

template <int S, int BN, bool TS>
__global__ void __launch_bounds__(I8_THREADS, 1)
    gemm_i8_kernel(const __grid_constant__ LaunchMaps pm,
                   const GemmJob *__restrict__ jobs, int njobs, int ntiles,
                   GemmList *list, unsigned *err) {
  i8_body<S, BN, true, TS>(&pm, jobs, njobs, ntiles, list, err);
}

template <int S, int BN, bool TS>
__global__ void __launch_bounds__(I8_THREADS, 1)
    gemm_i8_kernel_dm(const GemmJob *__restrict__ jobs, GemmList *list,
                      unsigned *err) {
  i8_body<S, BN, false, TS>(nullptr, jobs, list->njobs, list->ntiles, list,
                            err);
}

template <int S, int BN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(I8_THREADS, 1)
    gemm_i8_pair_kernel(const __grid_constant__ LaunchMaps pm,
                        const GemmJob *__restrict__ jobs, int njobs, int ntiles,
                        unsigned *err) {
  i8_pair_body<S, BN, true>(&pm, jobs, njobs, ntiles, err);
}

template <int S, int BN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(I8_THREADS, 1)
    gemm_i8_pair_kernel_dm(const GemmJob *__restrict__ jobs,
                           const GemmList *__restrict__ list, unsigned *err) {
  i8_pair_body<S, BN, false>(nullptr, jobs, list->njobs, list->ntiles, err);
}

template <typename K1, typename K2>
cudaError_t configure(K1 k1, K2 k2, int smem, bool &done) {
  if (done) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(
      k1, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
  if (e == cudaSuccess) done = true;
  return e;
}

template <int S, int BN, bool TS>
cudaError_t launch(const GemmJob *d_jobs, GemmList *d_list, int njobs,
                   int ntiles, const LaunchMaps *pm, int grid, unsigned *d_err,
                   cudaStream_t st) {
  using C = I8Cfg<S, BN, TS, false>;
  static bool configured = false;
  if (cudaError_t e = configure(gemm_i8_kernel<S, BN, TS>,
                                gemm_i8_kernel_dm<S, BN, TS>, C::SMEM,
                                configured))
    return e;
  if (pm)
    gemm_i8_kernel<S, BN, TS><<<grid, I8_THREADS, C::SMEM, st>>>(
        *pm, d_jobs, njobs, ntiles, d_list, d_err);
  else
    gemm_i8_kernel_dm<S, BN, TS><<<grid, I8_THREADS, C::SMEM, st>>>(
        d_jobs, d_list, d_err);
  return cudaGetLastError();
}

template <int S, int BN>
cudaError_t launch_pair(const GemmJob *d_jobs, const GemmList *d_list,
                        int njobs, int ntiles, const LaunchMaps *pm, int grid,
                        unsigned *d_err, cudaStream_t st) {
  using C = I8Cfg<S, BN, false, true>;
  static bool configured = false;
  if (cudaError_t e = configure(gemm_i8_pair_kernel<S, BN>,
                                gemm_i8_pair_kernel_dm<S, BN>, C::SMEM,
                                configured))
    return e;
  // one cluster (two CTAs) per pair tile, at most one CTA per SM
  int g = 2 * grid;
  if (g > GEMM_GRID) g = GEMM_GRID;
  g &= ~1;
  if (g < 2) g = 2;
  if (pm)
    gemm_i8_pair_kernel<S, BN><<<g, I8_THREADS, C::SMEM, st>>>(
        *pm, d_jobs, njobs, ntiles, d_err);
  else
    gemm_i8_pair_kernel_dm<S, BN><<<g, I8_THREADS, C::SMEM, st>>>(
        d_jobs, d_list, d_err);
  return cudaGetLastError();
}

// The tile variants of each slice count, the default (used when a plan does
// not tune) first, then narrower, CTA-pair, A-in-TMEM and two-stage forms.
// Every stage is one 64-byte K chunk.
constexpr I8Tile kTiles4[] = {{128, KB, 0, 0}, {64, KB, 0, 0},
                               {128, KB, 1, 0}, {112, KB, 0, 1}};
constexpr I8Tile kTiles5[] = {{96, KB, 0, 0}, {64, KB, 0, 0},
                               {96, KB, 1, 0}, {80, KB, 0, 1}};
constexpr I8Tile kTiles6[] = {{64, KB, 0, 0}, {64, KB, 0, 1}, {80, KB, 0, 0}};
constexpr I8Tile kTiles7[] = {{32, KB, 0, 0}};

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
                           GemmList *d_list, int njobs, int ntiles,
                           const LaunchMaps *pm, int grid, unsigned *d_err,
                           cudaStream_t st) {
  if (grid <= 0) return cudaSuccess;
  if (t.kc != KB) return cudaErrorInvalidValue;
#define PTB_I8(S_, BN_)                                                       \
  if (slices == S_ && t.bn == BN_ && !t.pair && !t.ts)                        \
    return launch<S_, BN_, false>(d_jobs, d_list, njobs, ntiles, pm, grid,   \
                                  d_err, st);
#define PTB_I8T(S_, BN_)                                                      \
  if (slices == S_ && t.bn == BN_ && !t.pair && t.ts)                         \
    return launch<S_, BN_, true>(d_jobs, d_list, njobs, ntiles, pm, grid,    \
                                 d_err, st);
#define PTB_I8P(S_, BN_)                                                      \
  if (slices == S_ && t.bn == BN_ && t.pair && !t.ts)                         \
    return launch_pair<S_, BN_>(d_jobs, d_list, njobs, ntiles, pm, grid,     \
                                d_err, st);
  PTB_I8(4, 128) PTB_I8(4, 64) PTB_I8P(4, 128) PTB_I8T(4, 112)
  PTB_I8(5, 96) PTB_I8(5, 64) PTB_I8P(5, 96) PTB_I8T(5, 80)
  PTB_I8(6, 64) PTB_I8T(6, 64) PTB_I8(6, 80)
  PTB_I8(7, 32)
#undef PTB_I8
#undef PTB_I8T
#undef PTB_I8P
  return cudaErrorInvalidValue;
}

}  // namespace ptb
