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
// contiguous in a or b (T[c][ab], U2, P) are staged through shared memory.
// Each CTA writes one partial sum; reduce_partials adds them in a fixed order.
#include "common.cuh"
#include "engine.h"

namespace ptb {

namespace {

__device__ __forceinline__ int64_t pairidx(int p, int q) {
  return (int64_t)p * (p - 1) / 2 + q;
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

// Disconnected term of a same-spin triple (src/pt.c:162-175).
__device__ __forceinline__ double disc_aaa(const double *ov, const double *g,
                                           int64_t gld, int o, int v, int i,
                                           int j, int k, int a, int b, int c) {
  const int64_t sl = (int64_t)v * gld;   // one [v][gld] slice of oovv
  const double *gjk = g + ((int64_t)j * o + k) * sl;
  const double *gik = g + ((int64_t)i * o + k) * sl;
  const double *gji = g + ((int64_t)j * o + i) * sl;
  const int64_t bc = (int64_t)b * gld + c, ac = (int64_t)a * gld + c,
                ba = (int64_t)b * gld + a;
  return ov[i * v + a] * gjk[bc] - ov[j * v + a] * gik[bc] -
         ov[k * v + a] * gji[bc] - ov[i * v + b] * gjk[ac] +
         ov[j * v + b] * gik[ac] + ov[k * v + b] * gji[ac] -
         ov[i * v + c] * gjk[ba] + ov[j * v + c] * gik[ba] +
         ov[k * v + c] * gji[ba];
}

template <bool FT>
__global__ void __launch_bounds__(EPI_THREADS)
    epi_aaa_kernel(const EpiArgs p) {
  extern __shared__ double sm[];
  // s3[a_][c_][b_] = T[c][pair(a,b)]  (and the R copy for (fT))
  double *s3 = sm;
  double *s3r = sm + EPI_A * EPI_C * EPI_PAD;

  const int4 tl = p.tiles[blockIdx.x];
  const int a0 = tl.x, b0 = tl.y, c0 = tl.z;
  const int t = blockIdx.y;
  const int i = p.trip[3 * t], j = p.trip[3 * t + 1], k = p.trip[3 * t + 2];
  const int v = p.va, o = p.oa;
  const double *base = p.ws + (int64_t)t * p.ws_stride;
  const double *T = base + p.offL[0];
  const double *R = FT ? base + p.offR[0] : nullptr;
  const int64_t ld = p.ld[0];

  for (int e = threadIdx.x; e < EPI_A * EPI_C * EPI_B; e += EPI_THREADS) {
    const int a_ = e / (EPI_C * EPI_B), c_ = (e / EPI_B) % EPI_C,
              b_ = e % EPI_B;
    const int a = a0 + a_, b = b0 + b_, c = c0 + c_;
    const bool ok = a < v && b < a && c < b;
    const int64_t off = (int64_t)c * ld + pairidx(a, b);
    s3[(a_ * EPI_C + c_) * EPI_PAD + b_] = ok ? T[off] : 0.0;
    if (FT) s3r[(a_ * EPI_C + c_) * EPI_PAD + b_] = ok ? R[off] : 0.0;
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = c0 + lane;
  double e = 0.0;
  for (int pr = warp; pr < EPI_A * EPI_B; pr += EPI_THREADS / 32) {
    const int a_ = pr / EPI_B, b_ = pr % EPI_B;
    const int a = a0 + a_, b = b0 + b_;
    if (!(a < v && b < a && c < b)) continue;
    const int64_t t1 = (int64_t)a * ld + pairidx(b, c);
    const int64_t t2 = (int64_t)b * ld + pairidx(a, c);
    const double w = T[t1] - T[t2] + s3[(a_ * EPI_C + lane) * EPI_PAD + b_];
    const double r =
        FT ? R[t1] - R[t2] + s3r[(a_ * EPI_C + lane) * EPI_PAD + b_] : w;
    const double x =
        disc_aaa(p.ov1_a, p.g1_aa, p.g1_ld_aa, o, v, i, j, k, a, b, c) +
        disc_aaa(p.ov2_a, p.g2_aa, p.g2_ld_aa, o, v, i, j, k, a, b, c);
    const double dn = p.d_a[i * v + a] + p.d_a[j * v + b] + p.d_a[k * v + c];
    e += (w - x) * r / dn;
  }
  const double s = block_sum(e);
  if (threadIdx.x == 0) p.partials[(int64_t)t * p.ntiles + blockIdx.x] = s;
}

// ---------------------------------------------------------------- aab ----

template <bool FT>
__global__ void __launch_bounds__(EPI_THREADS)
    epi_aab_kernel(const EpiArgs p) {
  extern __shared__ double sm[];
  constexpr int S = EPI_A * EPI_C * EPI_PAD;
  // sx[a_][c_][b_] = U2[a][c][b];  sy[b_][c_][a_] = U2[b][c][a];
  // sp[c_][a_][b_] = P[c][pair(a,b)]   (R copies follow for (fT))
  double *sx = sm, *sy = sm + S, *sp = sm + 2 * S;

  const int4 tl = p.tiles[blockIdx.x];
  const int a0 = tl.x, b0 = tl.y, c0 = blockIdx.y * EPI_C;
  const int t = blockIdx.z;
  const int i = p.trip[3 * t], j = p.trip[3 * t + 1], k = p.trip[3 * t + 2];
  const int oa = p.oa, va = p.va, ob = p.ob, vb = p.vb;
  const double *base = p.ws + (int64_t)t * p.ws_stride;
  const int64_t ld1 = p.ld[0], ld2 = p.ld[1], ldp = p.ld[2];
  const int64_t r1 = p.rowU1, r2 = p.rowU2;

#pragma unroll
  for (int side = 0; side < (FT ? 2 : 1); ++side) {
    const int64_t *off = side ? p.offR : p.offL;
    const double *U2 = base + off[1];
    const double *P = base + off[2];
    double *x_ = sx + side * 3 * S, *y_ = sy + side * 3 * S,
           *q_ = sp + side * 3 * S;
    for (int e = threadIdx.x; e < EPI_A * EPI_C * EPI_B; e += EPI_THREADS) {
      const int u = e / (EPI_C * EPI_B), c_ = (e / EPI_B) % EPI_C,
                w = e % EPI_B;
      const int c = c0 + c_;
      const bool cok = c < vb;
      {  // x_[u=a_][c_][w=b_] = U2[a][c][b]
        const int a = a0 + u, b = b0 + w;
        x_[(u * EPI_C + c_) * EPI_PAD + w] =
            (cok && a < va && b < va) ? U2[(int64_t)a * ld2 + c * r2 + b]
                                      : 0.0;
      }
      {  // y_[u=b_][c_][w=a_] = U2[b][c][a]
        const int b = b0 + u, a = a0 + w;
        y_[(u * EPI_C + c_) * EPI_PAD + w] =
            (cok && a < va && b < va) ? U2[(int64_t)b * ld2 + c * r2 + a]
                                      : 0.0;
      }
      {  // q_[c_][u=a_][w=b_] = P[c][pair(a,b)]
        const int a = a0 + u, b = b0 + w;
        q_[(c_ * EPI_A + u) * EPI_PAD + w] =
            (cok && a < va && b < a) ? P[(int64_t)c * ldp + pairidx(a, b)]
                                     : 0.0;
      }
    }
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = c0 + lane;
  const double *U1 = base + p.offL[0];
  const double *U1r = FT ? base + p.offR[0] : nullptr;
  // disconnected-term slices (src/pt.c:433-442)
  const double *g1jk = p.g1_ab + ((int64_t)j * ob + k) * va * p.g1_ld_ab;
  const double *g1ik = p.g1_ab + ((int64_t)i * ob + k) * va * p.g1_ld_ab;
  const double *g1ji = p.g1_aa + ((int64_t)j * oa + i) * va * p.g1_ld_aa;
  const double *g2jk = p.g2_ab + ((int64_t)j * ob + k) * va * p.g2_ld_ab;
  const double *g2ik = p.g2_ab + ((int64_t)i * ob + k) * va * p.g2_ld_ab;
  const double *g2ji = p.g2_aa + ((int64_t)j * oa + i) * va * p.g2_ld_aa;
  double e = 0.0;
  if (c < vb) {
    const double dk = p.d_b[k * vb + c];
    const double o1k = p.ov1_b[k * vb + c], o2k = p.ov2_b[k * vb + c];
    for (int pr = warp; pr < EPI_A * EPI_B; pr += EPI_THREADS / 32) {
      const int a_ = pr / EPI_B, b_ = pr % EPI_B;
      const int a = a0 + a_, b = b0 + b_;
      if (!(a < va && b < a)) continue;
      const int64_t u_ab = (int64_t)a * ld1 + b * r1 + c;
      const int64_t u_ba = (int64_t)b * ld1 + a * r1 + c;
      const int ix = (a_ * EPI_C + lane) * EPI_PAD + b_;
      const int iy = (b_ * EPI_C + lane) * EPI_PAD + a_;
      const int iq = (lane * EPI_A + a_) * EPI_PAD + b_;
      const double w = U1[u_ab] + sx[ix] - U1[u_ba] - sy[iy] + sp[iq];
      const double r =
          FT ? U1r[u_ab] + sx[3 * S + ix] - U1r[u_ba] - sy[3 * S + iy] +
                   sp[3 * S + iq]
             : w;
      const int64_t bc1 = (int64_t)b * p.g1_ld_ab + c,
                    ac1 = (int64_t)a * p.g1_ld_ab + c;
      const int64_t bc2 = (int64_t)b * p.g2_ld_ab + c,
                    ac2 = (int64_t)a * p.g2_ld_ab + c;
      const double x =
          p.ov1_a[i * va + a] * g1jk[bc1] - p.ov1_a[i * va + b] * g1jk[ac1] -
          p.ov1_a[j * va + a] * g1ik[bc1] + p.ov1_a[j * va + b] * g1ik[ac1] +
          o1k * g1ji[(int64_t)b * p.g1_ld_aa + a] +
          p.ov2_a[i * va + a] * g2jk[bc2] - p.ov2_a[i * va + b] * g2jk[ac2] -
          p.ov2_a[j * va + a] * g2ik[bc2] + p.ov2_a[j * va + b] * g2ik[ac2] +
          o2k * g2ji[(int64_t)b * p.g2_ld_aa + a];
      const double dn = p.d_a[i * va + a] + p.d_a[j * va + b] + dk;
      e += (w - x) * r / dn;
    }
  }
  const double s = block_sum(e);
  if (threadIdx.x == 0)
    p.partials[(int64_t)t * p.ntiles + blockIdx.y * gridDim.x + blockIdx.x] =
        s;
}

__global__ void __launch_bounds__(256)
    reduce_partials_kernel(const double *partials, int ntiles,
                           const int *slot, double *e_slot) {
  __shared__ double red[256];
  const int t = blockIdx.x;
  double s = 0.0;
  for (int x = threadIdx.x; x < ntiles; x += 256)
    s += partials[(int64_t)t * ntiles + x];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) e_slot[slot[t]] = red[0];
}

template <typename K>
cudaError_t set_smem(K kern, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)bytes);
}

}  // namespace

size_t epi_smem_bytes(bool aab, bool ft) {
  const size_t s = (size_t)EPI_A * EPI_C * EPI_PAD * sizeof(double);
  return (aab ? 3 : 1) * (ft ? 2 : 1) * s;
}

cudaError_t epi_aaa_launch(const EpiArgs &a, bool ft, int ntrip,
                           cudaStream_t st) {
  if (a.ntiles <= 0 || ntrip <= 0) return cudaSuccess;
  const size_t smem = epi_smem_bytes(false, ft);
  dim3 grid(a.ntiles, ntrip);
  cudaError_t e;
  if (ft) {
    if ((e = set_smem(epi_aaa_kernel<true>, smem)) != cudaSuccess) return e;
    epi_aaa_kernel<true><<<grid, EPI_THREADS, smem, st>>>(a);
  } else {
    if ((e = set_smem(epi_aaa_kernel<false>, smem)) != cudaSuccess) return e;
    epi_aaa_kernel<false><<<grid, EPI_THREADS, smem, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t epi_aab_launch(const EpiArgs &a, bool ft, int ntrip,
                           cudaStream_t st) {
  if (a.ntiles <= 0 || ntrip <= 0) return cudaSuccess;
  const size_t smem = epi_smem_bytes(true, ft);
  const int npairs = a.ntiles / a.ctiles;
  dim3 grid(npairs, a.ctiles, ntrip);
  cudaError_t e;
  if (ft) {
    if ((e = set_smem(epi_aab_kernel<true>, smem)) != cudaSuccess) return e;
    epi_aab_kernel<true><<<grid, EPI_THREADS, smem, st>>>(a);
  } else {
    if ((e = set_smem(epi_aab_kernel<false>, smem)) != cudaSuccess) return e;
    epi_aab_kernel<false><<<grid, EPI_THREADS, smem, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t reduce_partials_launch(const double *partials, int ntiles,
                                   int ntrip, const int *slot, double *e_slot,
                                   cudaStream_t st) {
  if (ntrip <= 0) return cudaSuccess;
  reduce_partials_kernel<<<ntrip, 256, 0, st>>>(partials, ntiles, slot,
                                                e_slot);
  return cudaGetLastError();
}

}  // namespace ptb
