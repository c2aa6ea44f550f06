// Energy epilogues: assemble W(abc) from a triple's contraction outputs,
// add the disconnected term and the denominator, and reduce the triple's
// energy (src/pt.c:291-295, 433-445 for (T); 697-700, 916-927 for (fT)).
//
// Same-spin triples (i<j<k):  one output T[x][pair] per amplitude, and
//   W[a>b>c] = T[a][bc] - T[b][ac] + T[c][ab]                (pair = p(p-1)/2+q)
// Mixed-spin triples (i<j alpha, k beta): outputs U1[x][y][c], U2[x][c][y],
// P[c][pair] per amplitude, and
//   W[a>b,c] = U1[a][b][c] + U2[a][c][b] - U1[b][a][c] - U2[b][c][a]
//              + P[c][ab].
// Energy per element: (W - X) * R / D with R = W for (T) and R = the right
// amplitude for (fT); X is the disconnected term, D the denominator.
//
// A CTA handles an 8 (a) x 8 (b) x 32 (c) tile of one triple; lanes run over
// c so the loads of U1/T rows are coalesced, and the operands that are
// contiguous in a or b (T[c][ab], U2, P) are staged through shared memory
// as [x][y][c] rows of EPI_CS = 34 doubles: the fill (8 consecutive y per
// 8 lanes) and the reads (32 consecutive c) are both free of bank conflicts.
// Each CTA tile writes one partial sum; reduce_partials adds them in a fixed
// order.  Launches are persistent: a fixed grid strides over the flat tiles
// of a device-memory item list (EpiList), whose items (triples) may belong
// to different plans; each item points at its spin case's fixed arguments,
// which a CTA copies to shared memory.
#include "common.cuh"
#include "engine.h"

namespace ptb {

namespace {

// CTAs per SM the energy kernels are compiled for (80 registers each): the
// kernels are latency-bound, and three CTAs of 256 threads keep more loads
// in flight than two (31 -> 40 % of DRAM peak measured), four spill.
constexpr int EPI_MINB = 3;

// Shared-memory layout (doubles) of the mixed-spin epilogue's staged
// disconnected-term slices, after its U2 / P staging: g1[j,k][b][c],
// g1[i,k][b][c] (EPI_B x EPI_C each), g1[j,i][b][a] (EPI_B x EPI_A), t1[i][b],
// t1[j][b], d[j][b] (EPI_B each), then the same for the f_ov half.
constexpr int EPI_SD_G1JK = 0, EPI_SD_G1IK = 256, EPI_SD_G1JI = 512,
              EPI_SD_T1I = 576, EPI_SD_T1J = 584, EPI_SD_DJ = 592,
              EPI_SD_G2JK = 600, EPI_SD_G2IK = 856, EPI_SD_G2JI = 1112,
              EPI_SD_F1I = 1176, EPI_SD_F1J = 1184, EPI_SD_SIZE = 1192;
static_assert(EPI_THREADS == EPI_B * EPI_C && EPI_B * EPI_C == 256 &&
                  EPI_A * EPI_B == 64 && EPI_A == 8 && EPI_B == 8,
              "one staged (b, c) per thread; offsets above");

__device__ __forceinline__ int64_t pairidx(int p, int q) {
  return (int64_t)p * (p - 1) / 2 + q;
}

__device__ __forceinline__ int pair32(int p, int q) {
  return p * (p - 1) / 2 + q;
}

// Fixed-order block reduction of one double per thread.
__device__ double block_sum(double x) {
  __shared__ double red[EPI_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < EPI_THREADS / 32; ++i) s += red[i];
  return s;
}

// ---------------------------------------------------------------- aaa ----

// Thread layout of both epilogues: warp w handles a = a0 + w, lane l handles
// c = c0 + l, and each thread walks the tile's 8 values of b (unrolled,
// branch-free with clamped indices and a validity mask, so the loads of
// several b are in flight together).

// 8-byte asynchronous global -> shared copy; ok == false writes 0.0 (the
// source is not read: src-size 0 zero-fills the destination).
__device__ __forceinline__ void cp_async8(double *dst, const double *src,
                                          bool ok) {
  asm volatile(
      "cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(ok ? 8 : 0)
      : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::
                   : "memory");
}

// A persistent CTA's walk over the items of an EpiList, kept in shared
// memory (no registers live across tiles): its tiles come in increasing
// order and an item spans many of them, so the binary search (a chain of
// dependent global loads) runs only when a tile leaves the current item, and
// the case arguments are copied to shared memory only when they change
// (items of one spin case of one plan share them).  Thread 0 advances it
// before the barrier that ends a tile.
struct ItemWalk {
  int cur, next_begin;          // item index; first tile of the next item
  const EpiArgs *staged;        // whose arguments shared memory holds
  __device__ __forceinline__ void seek(const EpiList *l, int blk) {
    if (blk < next_begin) return;
    cur = find_entry(l->items, l->nitems, blk, &EpiItem::block_begin);
    next_begin = cur + 1 < l->nitems ? l->items[cur + 1].block_begin
                                     : 0x7fffffff;
  }
};

// Copies an item's case arguments into shared memory (all threads).
__device__ __forceinline__ void load_args(EpiArgs &dst, const EpiArgs *src) {
  static_assert(sizeof(EpiArgs) % 8 == 0, "8-byte words");
  constexpr int W = (int)(sizeof(EpiArgs) / 8);
  for (int x = threadIdx.x; x < W; x += blockDim.x)
    reinterpret_cast<long long *>(&dst)[x] =
        reinterpret_cast<const long long *>(src)[x];
  __syncthreads();
}

template <bool FT, bool LOOP, bool HASF>
__global__ void __launch_bounds__(EPI_THREADS, EPI_MINB)
    epi_aaa_kernel(const EpiList *__restrict__ list,
                   const EpiItem *__restrict__ items) {
  extern __shared__ double sm[];
  __shared__ EpiArgs p;
  constexpr int S = EPI_A * EPI_B * EPI_CS;
  constexpr int NIT = EPI_A * EPI_C * EPI_B / EPI_THREADS;
  // s3[a_][b_][c_] = T[c][pair(a,b)]  (the R copy follows for (fT))
  double *s3 = sm;
  // LOOP: a fixed grid striding over the flat tiles of all items; else one
  // CTA per (tile, item) of a 2-D grid
  int blk = blockIdx.x;
  if (LOOP && blk >= list->nblocks) return;
  __shared__ ItemWalk walk;
  if (LOOP) {
    if (threadIdx.x == 0) {
      walk.next_begin = 0;
      walk.staged = nullptr;
      walk.seek(list, blk);
    }
    __syncthreads();
  }
  do {
  const EpiItem &item = LOOP ? list->items[walk.cur] : items[blockIdx.y];
  const int local = LOOP ? blk - item.block_begin : blk;
  if (!LOOP && local >= item.nblk) return;
  if (!LOOP || item.args != walk.staged) {   // uniform over the CTA
    load_args(p, item.args);   // ends with a barrier
    if (LOOP && threadIdx.x == 0) walk.staged = item.args;
  }
  const int4 tl = p.tiles[local];
  const int a0 = tl.x, b0 = tl.y, c0 = tl.z;
  const int i = item.i, j = item.j, k = item.k;
  const int v = p.va, o = p.oa;
  const bool has_f = HASF && p.has_f != 0;   // HASF false: f_ov is zero
  const int g1l = (int)p.g1_ld_aa, g2l = (int)p.g2_ld_aa;
  const double *base = item.ws;
  const double *T = base + p.offL[0];
  const double *R = FT ? base + p.offR[0] : nullptr;
  const int64_t ld = p.ld[0];
  const int ldi = (int)ld;

  // stage T[c][pair(a,b)] asynchronously; its wait comes after the loads
  // of the per-thread operands below, so both latencies overlap
#pragma unroll
  for (int it = 0; it < NIT; ++it) {
    const int e = threadIdx.x + it * EPI_THREADS;
    const int a_ = e / (EPI_C * EPI_B), c_ = (e / EPI_B) % EPI_C,
              b_ = e % EPI_B;
    const int a = a0 + a_, b = b0 + b_, c = c0 + c_;
    const bool ok = a < v && b < a && c < b;
    const int64_t off = ok ? (int64_t)c * ld + pairidx(a, b) : 0;
    const int idx = (a_ * EPI_B + b_) * EPI_CS + c_;
    cp_async8(&s3[idx], T + off, ok);
    if (FT) cp_async8(&s3[S + idx], R + off, ok);
  }

  const int a_ = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = a0 + a_, c = c0 + lane;
  const int ac = a < v ? a : v - 1;       // clamped indices for addressing
  const int cc = c < v ? c : v - 1;
  // disconnected term (src/pt.c:162-175): the parts that depend on (a, c)
  const int64_t sl1 = (int64_t)v * p.g1_ld_aa, sl2 = (int64_t)v * p.g2_ld_aa;
  const double *g1jk = p.g1_aa + ((int64_t)j * o + k) * sl1;
  const double *g1ik = p.g1_aa + ((int64_t)i * o + k) * sl1;
  const double *g1ji = p.g1_aa + ((int64_t)j * o + i) * sl1;
  const double *g2jk = p.g2_aa + ((int64_t)j * o + k) * sl2;
  const double *g2ik = p.g2_aa + ((int64_t)i * o + k) * sl2;
  const double *g2ji = p.g2_aa + ((int64_t)j * o + i) * sl2;
  const double *u1 = p.ov1_a, *u2 = p.ov2_a;
  const int64_t ac1 = (int64_t)ac * p.g1_ld_aa + cc,
                ac2 = (int64_t)ac * p.g2_ld_aa + cc;
  const double A1jk = g1jk[ac1], A1ik = g1ik[ac1], A1ji = g1ji[ac1];
  const double A2jk = g2jk[ac2], A2ik = g2ik[ac2], A2ji = g2ji[ac2];
  const double t1ia = u1[i * v + ac], t1ja = u1[j * v + ac],
               t1ka = u1[k * v + ac];
  const double t1ic = u1[i * v + cc], t1jc = u1[j * v + cc],
               t1kc = u1[k * v + cc];
  const double f_ia = u2[i * v + ac], f_ja = u2[j * v + ac],
               f_ka = u2[k * v + ac];
  const double f_ic = u2[i * v + cc], f_jc = u2[j * v + cc],
               f_kc = u2[k * v + cc];
  const double dia = p.d_a[i * v + ac], dkc = p.d_a[k * v + cc];
  cp_async_wait_all();
  __syncthreads();

  // one b at a time: the element's energy is added as soon as its operands
  // are in (arrays of all 8 b values spilled registers); the loop is
  // unrolled so the loads of later b overlap the arithmetic of earlier ones
  double e = 0.0;
#pragma unroll
  for (int b_ = 0; b_ < EPI_B; ++b_) {
    const int b = b0 + b_;
    const bool ok = a < v && b < a && c < b;
    const int bc = b < v ? b : v - 1;
    const int cb = ok ? c : 0;               // pair index needs c < b
    const int t1 = ac * ldi + pair32(bc, cb);   // < 2^31 (plan check)
    const int t2 = bc * ldi + pair32(ac, cb);
    const int is = (a_ * EPI_B + b_) * EPI_CS + lane;
    const double w = T[t1] - T[t2] + s3[is];
    const double rr = FT ? R[t1] - R[t2] + s3[S + is] : w;
    const int bc1 = bc * g1l + cc, bc2 = bc * g2l + cc;
    const int ba1 = bc * g1l + ac, ba2 = bc * g2l + ac;
    // the 9-term sums of src/pt.c:166-174 for (t1, i_oovv) and (f_ov, t2);
    // the second is skipped when f_ov is zero (its terms would all be 0)
    double x =
        t1ia * g1jk[bc1] - t1ja * g1ik[bc1] - t1ka * g1ji[bc1] -
        u1[i * v + bc] * A1jk + u1[j * v + bc] * A1ik +
        u1[k * v + bc] * A1ji - t1ic * g1jk[ba1] + t1jc * g1ik[ba1] +
        t1kc * g1ji[ba1];
    if (has_f)
      x += f_ia * g2jk[bc2] - f_ja * g2ik[bc2] - f_ka * g2ji[bc2] -
           u2[i * v + bc] * A2jk + u2[j * v + bc] * A2ik +
           u2[k * v + bc] * A2ji - f_ic * g2jk[ba2] + f_jc * g2ik[ba2] +
           f_kc * g2ji[ba2];
    const double dd = (dia + p.d_a[j * v + bc]) + dkc;
    if (ok) e += (w - x) * rr * recip_nr(dd);
  }
  const double s = block_sum(e);
  if (threadIdx.x == 0) item.partials[local] = s;
  if (!LOOP) break;
  blk += gridDim.x;
  if (threadIdx.x == 0) walk.seek(list, blk);
  __syncthreads();   // shared memory is refilled by the next tile
  } while (blk < list->nblocks);
}

// ---------------------------------------------------------------- aab ----

template <bool FT, bool LOOP, bool HASF>
__global__ void __launch_bounds__(EPI_THREADS, EPI_MINB)
    epi_aab_kernel(const EpiList *__restrict__ list,
                   const EpiItem *__restrict__ items) {
  extern __shared__ double sm[];
  __shared__ EpiArgs p;
  constexpr int S = EPI_A * EPI_B * EPI_CS;
  constexpr int NIT = EPI_A * EPI_C * EPI_B / EPI_THREADS;
  // sx[a_][b_][c_] = U2[a][c][b];  sy[b_][a_][c_] = U2[b][c][a];
  // sp[a_][b_][c_] = P[c][pair(a,b)]   (R copies follow for (fT))
  double *sx = sm, *sy = sm + S, *sp = sm + 2 * S;
  // LOOP: a fixed grid striding over the flat tiles of all items; else one
  // CTA per (tile, item) of a 2-D grid
  int blk = blockIdx.x;
  if (LOOP && blk >= list->nblocks) return;
  __shared__ ItemWalk walk;
  if (LOOP) {
    if (threadIdx.x == 0) {
      walk.next_begin = 0;
      walk.staged = nullptr;
      walk.seek(list, blk);
    }
    __syncthreads();
  }
  do {
  const EpiItem &item = LOOP ? list->items[walk.cur] : items[blockIdx.y];
  const int local = LOOP ? blk - item.block_begin : blk;
  if (!LOOP && local >= item.nblk) return;
  if (!LOOP || item.args != walk.staged) {   // uniform over the CTA
    load_args(p, item.args);   // ends with a barrier
    if (LOOP && threadIdx.x == 0) walk.staged = item.args;
  }
  const int npairs = p.ntiles / p.ctiles;   // tiles: c block major
  // the (a, b) tiles are the triangle a0 = 8t, b0 = 8u, u <= t, in row
  // order (the last row may stop at u = t - 1); tile L sits in row
  // t = floor((sqrt(8L + 1) - 1) / 2), computed here instead of loaded from
  // the case's tile table, so the data loads need one dependent load less
  const int L = local % npairs;
  int t = (int)((sqrtf(8.0f * (float)L + 1.0f) - 1.0f) * 0.5f);
  while ((t + 1) * (t + 2) / 2 <= L) ++t;
  while (t * (t + 1) / 2 > L) --t;
  const int a0 = EPI_A * t, b0 = EPI_B * (L - t * (t + 1) / 2);
  const int c0 = (local / npairs) * EPI_C;
  const int i = item.i, j = item.j, k = item.k;
  const int oa = p.oa, va = p.va, ob = p.ob, vb = p.vb;
  const double *base = item.ws;
  const int64_t ld2 = p.ld[1], ldp = p.ld[2];
  const int64_t r2 = p.rowU2;
  // 32-bit strides for the per-element loop (the plan keeps a triple's
  // arrays and the i_oovv / amplitude slices under 2^31 elements)
  const int ld1 = (int)p.ld[0], r1 = (int)p.rowU1;
  const int g1lab = (int)p.g1_ld_ab, g2lab = (int)p.g2_ld_ab;
  const int g1laa = (int)p.g1_ld_aa, g2laa = (int)p.g2_ld_aa;
  const bool has_f = HASF && p.has_f != 0;   // HASF false: f_ov is zero

  // stage U2 (both orientations) and P asynchronously; the wait comes after
  // the per-thread operand loads below
#pragma unroll
  for (int side = 0; side < (FT ? 2 : 1); ++side) {
    const int64_t *off = side ? p.offR : p.offL;
    const double *U2 = base + off[1];
    const double *P = base + off[2];
#pragma unroll
    for (int it = 0; it < NIT; ++it) {
      const int e = threadIdx.x + it * EPI_THREADS;
      const int u = e / (EPI_C * EPI_B), c_ = (e / EPI_B) % EPI_C,
                w = e % EPI_B;
      const int c = c0 + c_;
      const bool cok = c < vb;
      const int idx = side * 3 * S + (u * EPI_B + w) * EPI_CS + c_;
      const int ax = a0 + u, bx = b0 + w;     // x: U2[a][c][b]
      const bool okx = cok && ax < va && bx < va;
      cp_async8(&sx[idx], U2 + (okx ? (int64_t)ax * ld2 + c * r2 + bx : 0),
                okx);
      const int by = b0 + u, ay = a0 + w;     // y: U2[b][c][a]
      const bool oky = cok && ay < va && by < va;
      cp_async8(&sy[idx], U2 + (oky ? (int64_t)by * ld2 + c * r2 + ay : 0),
                oky);
      const bool okp = cok && ax < va && bx < ax;   // p: P[c][pair(a,b)]
      cp_async8(&sp[idx],
                P + (okp ? (int64_t)c * ldp + pairidx(ax, bx) : 0), okp);
    }
  }

  const int a_ = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = a0 + a_, c = c0 + lane;
  const int ac = a < va ? a : va - 1, cc = c < vb ? c : vb - 1;
  const double *U1 = base + p.offL[0];
  const double *U1r = FT ? base + p.offR[0] : nullptr;
  // disconnected-term slices (src/pt.c:433-442)
  const double *g1jk = p.g1_ab + ((int64_t)j * ob + k) * va * p.g1_ld_ab;
  const double *g1ik = p.g1_ab + ((int64_t)i * ob + k) * va * p.g1_ld_ab;
  const double *g1ji = p.g1_aa + ((int64_t)j * oa + i) * va * p.g1_ld_aa;
  const double *g2jk = p.g2_ab + ((int64_t)j * ob + k) * va * p.g2_ld_ab;
  const double *g2ik = p.g2_ab + ((int64_t)i * ob + k) * va * p.g2_ld_ab;
  const double *g2ji = p.g2_aa + ((int64_t)j * oa + i) * va * p.g2_ld_aa;
  const double *u1 = p.ov1_a, *u2 = p.ov2_a;
  // The parts of the disconnected term that vary with b -- g[b][c] rows,
  // g[b][a], and the per-b amplitudes and denominators -- are the same for
  // every warp (a) of the tile: staged once into shared memory (zero where
  // b or c is outside the space; those elements are masked) instead of
  // loaded by each warp in the b loop.
  double *sd = sm + (FT ? 6 : 3) * S;
  {
    const int t = threadIdx.x;   // one (b, c) per thread
    const int bt = b0 + (t >> 5), ct = c0 + (t & 31);
    const bool okbc = bt < va && ct < vb;
    cp_async8(&sd[EPI_SD_G1JK + t], g1jk + (okbc ? bt * g1lab + ct : 0), okbc);
    cp_async8(&sd[EPI_SD_G1IK + t], g1ik + (okbc ? bt * g1lab + ct : 0), okbc);
    if (has_f) {
      cp_async8(&sd[EPI_SD_G2JK + t], g2jk + (okbc ? bt * g2lab + ct : 0),
                okbc);
      cp_async8(&sd[EPI_SD_G2IK + t], g2ik + (okbc ? bt * g2lab + ct : 0),
                okbc);
    }
    if (t < EPI_B * EPI_A) {   // (b, a) of g[j][i]
      const int bb = b0 + (t >> 3), aa = a0 + (t & 7);
      const bool okba = bb < va && aa < va;
      cp_async8(&sd[EPI_SD_G1JI + t], g1ji + (okba ? bb * g1laa + aa : 0),
                okba);
      if (has_f)
        cp_async8(&sd[EPI_SD_G2JI + t], g2ji + (okba ? bb * g2laa + aa : 0),
                  okba);
    } else if (t < EPI_B * EPI_A + EPI_B) {   // per b
      const int b_ = t - EPI_B * EPI_A, bb = b0 + b_;
      const bool okb = bb < va;
      cp_async8(&sd[EPI_SD_T1I + b_], u1 + (okb ? i * va + bb : 0), okb);
      cp_async8(&sd[EPI_SD_T1J + b_], u1 + (okb ? j * va + bb : 0), okb);
      cp_async8(&sd[EPI_SD_DJ + b_], p.d_a + (okb ? j * va + bb : 0), okb);
      if (has_f) {
        cp_async8(&sd[EPI_SD_F1I + b_], u2 + (okb ? i * va + bb : 0), okb);
        cp_async8(&sd[EPI_SD_F1J + b_], u2 + (okb ? j * va + bb : 0), okb);
      }
    }
  }
  const int64_t ac1 = (int64_t)ac * p.g1_ld_ab + cc,
                ac2 = (int64_t)ac * p.g2_ld_ab + cc;
  const double A1jk = g1jk[ac1], A1ik = g1ik[ac1];
  const double A2jk = g2jk[ac2], A2ik = g2ik[ac2];
  const double t1ia = u1[i * va + ac], t1ja = u1[j * va + ac];
  const double f_ia = u2[i * va + ac], f_ja = u2[j * va + ac];
  const double o1k = p.ov1_b[k * vb + cc], o2k = p.ov2_b[k * vb + cc];
  const double dia = p.d_a[i * va + ac], dkc = p.d_b[k * vb + cc];
  // U1 in both orientations, loaded before the wait for the staged
  // operands so that the two sets of loads are in flight together (the
  // wait is a memory barrier for the compiler)
  double xu[EPI_B];
#pragma unroll
  for (int b_ = 0; b_ < EPI_B; ++b_) {
    const int bc = b0 + b_ < va ? b0 + b_ : va - 1;
    xu[b_] = U1[ac * ld1 + bc * r1 + cc] - U1[bc * ld1 + ac * r1 + cc];
  }   // offsets < 2^31 (checked by the plan)
  cp_async_wait_all();
  __syncthreads();

  // one b at a time (see the same-spin kernel)
  double e = 0.0;
#pragma unroll
  for (int b_ = 0; b_ < EPI_B; ++b_) {
    const int b = b0 + b_;
    const bool ok = a < va && b < a && c < vb;
    const int bc = b < va ? b : va - 1;
    const int u_ab = ac * ld1 + bc * r1 + cc;
    const int u_ba = bc * ld1 + ac * r1 + cc;
    const int ix = (a_ * EPI_B + b_) * EPI_CS + lane;
    const int iy = (b_ * EPI_A + a_) * EPI_CS + lane;
    const double w = xu[b_] + sx[ix] - sy[iy] + sp[ix];
    const double rr = FT ? U1r[u_ab] + sx[3 * S + ix] - U1r[u_ba] -
                               sy[3 * S + iy] + sp[3 * S + ix]
                         : w;
    const int bcl = b_ * EPI_C + lane, ba = b_ * EPI_A + a_;
    double x = t1ia * sd[EPI_SD_G1JK + bcl] - sd[EPI_SD_T1I + b_] * A1jk -
               t1ja * sd[EPI_SD_G1IK + bcl] + sd[EPI_SD_T1J + b_] * A1ik +
               o1k * sd[EPI_SD_G1JI + ba];
    if (has_f)   // the (f_ov, t2) half, zero when f_ov is
      x += f_ia * sd[EPI_SD_G2JK + bcl] - sd[EPI_SD_F1I + b_] * A2jk -
           f_ja * sd[EPI_SD_G2IK + bcl] + sd[EPI_SD_F1J + b_] * A2ik +
           o2k * sd[EPI_SD_G2JI + ba];
    const double dd = (dia + sd[EPI_SD_DJ + b_]) + dkc;
    if (ok) e += (w - x) * rr * recip_nr(dd);
  }
  const double s = block_sum(e);
  if (threadIdx.x == 0) item.partials[local] = s;
  if (!LOOP) break;
  blk += gridDim.x;
  if (threadIdx.x == 0) walk.seek(list, blk);
  __syncthreads();   // shared memory is refilled by the next tile
  } while (blk < list->nblocks);
}

__global__ void __launch_bounds__(256)
    reduce_partials_kernel(const RedList *__restrict__ list) {
  __shared__ double red[256];
  const int nitems = list->nitems;
  for (int t = blockIdx.x; t < nitems; t += gridDim.x) {
    const RedItem it = list->items[t];
    double s = 0.0;
    for (int x = threadIdx.x; x < it.n; x += 256) s += it.partials[x];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) *it.dst = red[0];
    __syncthreads();
  }
}

template <typename K>
cudaError_t set_smem(K kern, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)bytes);
}

template <typename K>
cudaError_t launch_epi(K kern, const EpiList *d_list, const EpiItem *d_items,
                       size_t smem, dim3 grid, cudaStream_t st) {
  cudaError_t e = set_smem(kern, smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, EPI_THREADS, smem, st>>>(d_list, d_items);
  return cudaGetLastError();
}

}  // namespace

size_t epi_smem_bytes(bool aab, bool ft) {
  const size_t s = (size_t)EPI_A * EPI_B * EPI_CS * sizeof(double);
  return (aab ? 3 : 1) * (ft ? 2 : 1) * s +
         (aab ? EPI_SD_SIZE * sizeof(double) : 0);
}

int epi_blocks_per_sm(bool aab, bool ft) {
  const size_t smem = epi_smem_bytes(aab, ft);
  int n = 0;
  cudaError_t e;
  if (aab) {
    if (ft) {
      set_smem(epi_aab_kernel<true, true, true>, smem);
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &n, epi_aab_kernel<true, true, true>, EPI_THREADS, smem);
    } else {
      set_smem(epi_aab_kernel<false, true, true>, smem);
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &n, epi_aab_kernel<false, true, true>, EPI_THREADS, smem);
    }
  } else {
    if (ft) {
      set_smem(epi_aaa_kernel<true, true, true>, smem);
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &n, epi_aaa_kernel<true, true, true>, EPI_THREADS, smem);
    } else {
      set_smem(epi_aaa_kernel<false, true, true>, smem);
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &n, epi_aaa_kernel<false, true, true>, EPI_THREADS, smem);
    }
  }
  return (e == cudaSuccess && n > 0) ? n : 1;
}

// Persistent launches (fixed grids, graph replays) use the general kernels;
// direct launches whose items all have a zero f_ov (hasf false) use the
// kernels compiled without the f_ov terms.
cudaError_t epi_aaa_launch(const EpiList *d_list, const EpiItem *d_items,
                           bool ft, bool hasf, int grid, int nitems,
                           bool persistent, cudaStream_t st) {
  if (grid <= 0 || nitems <= 0) return cudaSuccess;
  if (!persistent && !d_items) return cudaErrorInvalidValue;
  const size_t smem = epi_smem_bytes(false, ft);
  const dim3 g(grid, persistent ? 1 : nitems);
  if (persistent)
    return ft ? launch_epi(epi_aaa_kernel<true, true, true>, d_list, d_items, smem, g, st)
              : launch_epi(epi_aaa_kernel<false, true, true>, d_list, d_items, smem, g, st);
  if (hasf)
    return ft ? launch_epi(epi_aaa_kernel<true, false, true>, d_list, d_items, smem, g, st)
              : launch_epi(epi_aaa_kernel<false, false, true>, d_list, d_items, smem, g, st);
  return ft ? launch_epi(epi_aaa_kernel<true, false, false>, d_list, d_items, smem, g, st)
            : launch_epi(epi_aaa_kernel<false, false, false>, d_list, d_items, smem, g, st);
}

cudaError_t epi_aab_launch(const EpiList *d_list, const EpiItem *d_items,
                           bool ft, bool hasf, int grid, int nitems,
                           bool persistent, cudaStream_t st) {
  if (grid <= 0 || nitems <= 0) return cudaSuccess;
  if (!persistent && !d_items) return cudaErrorInvalidValue;
  const size_t smem = epi_smem_bytes(true, ft);
  const dim3 g(grid, persistent ? 1 : nitems);
  if (persistent)
    return ft ? launch_epi(epi_aab_kernel<true, true, true>, d_list, d_items, smem, g, st)
              : launch_epi(epi_aab_kernel<false, true, true>, d_list, d_items, smem, g, st);
  if (hasf)
    return ft ? launch_epi(epi_aab_kernel<true, false, true>, d_list, d_items, smem, g, st)
              : launch_epi(epi_aab_kernel<false, false, true>, d_list, d_items, smem, g, st);
  return ft ? launch_epi(epi_aab_kernel<true, false, false>, d_list, d_items, smem, g, st)
            : launch_epi(epi_aab_kernel<false, false, false>, d_list, d_items, smem, g, st);
}

cudaError_t reduce_partials_launch(const RedList *d_list, int grid,
                                   cudaStream_t st) {
  if (grid <= 0) return cudaSuccess;
  reduce_partials_kernel<<<grid, 256, 0, st>>>(d_list);
  return cudaGetLastError();
}

}  // namespace ptb
