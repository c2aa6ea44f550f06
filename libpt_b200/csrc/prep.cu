// Operand preparation: copy pt.h blocks into the engine's padded layout.
//
// Every GEMM operand block keeps the pt.h index order but has its innermost
// dimension padded to a multiple of 4 doubles (32 bytes) with zeros, so that
// TMA views with 32-byte-wide boxes can address any row; the packed-pair
// copy of same-spin amplitudes feeds the OOVO contractions of same-spin
// triples with columns indexed like the packed OVVV block (src/pt.h:51-52).
#include "common.cuh"
#include "engine.h"

namespace ptb {

namespace {

template <typename T>
__global__ void repack_kernel(const T *__restrict__ src, double *__restrict__ dst,
                              int64_t rows, int64_t w, int64_t dpitch) {
  const int64_t total = rows * dpitch;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = x / dpitch, c = x - r * dpitch;
    dst[x] = c < w ? (double)src[r * w + c] : 0.0;
  }
}

__global__ void pack_pairs_kernel(const double *__restrict__ tau,
                                  double *__restrict__ out, int64_t npq, int v,
                                  int64_t ldv, int64_t ldp) {
  const int64_t total = npq * ldp;
  const int64_t np = (int64_t)v * (v - 1) / 2;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pq = x / ldp, n = x - pq * ldp;
    double val = 0.0;
    if (n < np) {
      // invert n = a(a-1)/2 + b, a > b >= 0
      int64_t a = (int64_t)((1.0 + sqrt(1.0 + 8.0 * (double)n)) * 0.5);
      while (a * (a - 1) / 2 > n) --a;
      while ((a + 1) * a / 2 <= n) ++a;
      const int64_t b = n - a * (a - 1) / 2;
      val = tau[(pq * v + a) * ldv + b];
    }
    out[x] = val;
  }
}

// TF32 hi/lo split of an FP32 value: hi is x rounded to TF32 (cvt.rna),
// lo = x - hi exactly; hi*hi + hi*lo + lo*hi reproduces products to about
// FP32 accuracy.
__device__ __forceinline__ void tf32_split(float x, float &hi, float &lo) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  hi = __uint_as_float(h);
  lo = x - hi;
}

// A side: elementwise split of a padded FP64 block (values exact in FP32).
__global__ void split_tf32_kernel(const double *__restrict__ src,
                                  float *__restrict__ hi,
                                  float *__restrict__ lo, int64_t n) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n;
       x += (int64_t)gridDim.x * blockDim.x) {
    float h, l;
    tf32_split((float)src[x], h, l);
    hi[x] = h;
    lo[x] = l;
  }
}

// B side: src[P][K][ldn] (FP64, N contiguous) -> dst[P][N][ldk] (K
// contiguous), split into TF32 hi/lo planes; 32x32 tiles through smem.
__global__ void transpose_split_tf32_kernel(const double *__restrict__ src,
                                            float *__restrict__ hi,
                                            float *__restrict__ lo, int K,
                                            int64_t N, int64_t ldn,
                                            int64_t ldk) {
  __shared__ float t[32][33];
  const int64_t p = blockIdx.z;
  const int64_t n0 = (int64_t)blockIdx.x * 32;
  const int k0 = blockIdx.y * 32;
  const double *s = src + p * K * ldn;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r;
    const int64_t n = n0 + threadIdx.x;
    t[r][threadIdx.x] = (k < K && n < N) ? (float)s[(int64_t)k * ldn + n] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t n = n0 + r;
    const int k = k0 + threadIdx.x;
    if (n < N && k < ldk) {
      float h, l;
      tf32_split(t[threadIdx.x][r], h, l);
      const int64_t o = (p * N + n) * ldk + k;
      hi[o] = h;
      lo[o] = l;
    }
  }
}

int grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t repack_launch(const void *src, bool src_fp32, double *dst,
                          int64_t rows, int64_t w, int64_t dpitch,
                          cudaStream_t st) {
  if (rows <= 0 || dpitch <= 0) return cudaSuccess;
  const int g = grid_for(rows * dpitch);
  if (src_fp32)
    repack_kernel<float><<<g, 256, 0, st>>>(static_cast<const float *>(src),
                                            dst, rows, w, dpitch);
  else
    repack_kernel<double><<<g, 256, 0, st>>>(static_cast<const double *>(src),
                                             dst, rows, w, dpitch);
  return cudaGetLastError();
}

cudaError_t pack_pairs_launch(const double *tau, double *out, int64_t npq,
                              int v, int64_t ldv, int64_t ldp,
                              cudaStream_t st) {
  if (npq <= 0 || ldp <= 0) return cudaSuccess;
  pack_pairs_kernel<<<grid_for(npq * ldp), 256, 0, st>>>(tau, out, npq, v, ldv,
                                                         ldp);
  return cudaGetLastError();
}

}  // namespace ptb

namespace ptb {

cudaError_t split_tf32_launch(const double *src, float *hi, float *lo,
                              int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  split_tf32_kernel<<<grid_for(n), 256, 0, st>>>(src, hi, lo, n);
  return cudaGetLastError();
}

cudaError_t transpose_split_tf32_launch(const double *src, float *hi,
                                        float *lo, int64_t P, int K,
                                        int64_t N, int64_t ldn, int64_t ldk,
                                        cudaStream_t st) {
  if (P <= 0 || N <= 0 || ldk <= 0) return cudaSuccess;
  for (int64_t p0 = 0; p0 < P; p0 += 65535) {
    const int64_t np = P - p0 < 65535 ? P - p0 : 65535;
    dim3 grid((unsigned)((N + 31) / 32), (unsigned)((ldk + 31) / 32),
              (unsigned)np);
    transpose_split_tf32_kernel<<<grid, dim3(32, 8), 0, st>>>(
        src + p0 * K * ldn, hi + p0 * N * ldk, lo + p0 * N * ldk, K, N, ldn,
        ldk);
  }
  return cudaGetLastError();
}

}  // namespace ptb

// ---- emulated FP64: power-of-two scales and digit planes ----------------
//
// An operand value a with scale exponent e (chosen per A row / B column as
// ceil-log2(max |a|) + 1, so |a 2^-e| < 1/2) is written in S base-2^b digits
//   a * 2^-e = sum_{p=1..S} d_p 2^-bp + remainder,
// every step exact in FP64 (Ozaki-style slicing).  Two digit forms:
//   b = 7: balanced digits |d_p| <= 64, each rounded to nearest from the
//          running remainder (|remainder| <= 2^-7S / 2); any first S' of the
//          S digits are the S'-digit decomposition.
//   b = 8: balanced digits of base 2^8, value 2 sum_p d_p 2^-8p: the top
//          digit rint(128 s) in [-64, 64], each lower digit rint(256 r) of
//          the running remainder, a digit 128 replaced by -128 with a carry
//          of 1 into the digit above (the top digit then stays <= 65), so
//          every digit fits a signed byte, |remainder| <= 2^-8S (in units
//          of s) and the truncation is unbiased; 8 bits of the operand per
//          lower plane instead of 7.  A prefix of S' digits is the S'-digit
//          decomposition but where a carry from below changed its last
//          digit (its error then stays within 2^-8S' (1 + 2^-7)).

namespace ptb {

namespace {

__device__ __forceinline__ void atomic_max_pos(unsigned long long *m,
                                               double x) {
  // non-negative doubles order like their bit patterns
  atomicMax(m, (unsigned long long)__double_as_longlong(x));
}

// rmax[x] = max over (pq, k < K) |src[pq][x][k]|, src rows padded to kp.
__global__ void rowmax_kernel(const double *__restrict__ src, int64_t npq,
                              int64_t R, int64_t K, int64_t kp,
                              unsigned long long *rmax) {
  const int64_t rows = npq * R;
  const int lane = threadIdx.x & 31;
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32;
       r < rows; r += ((int64_t)gridDim.x * blockDim.x) / 32) {
    double m = 0.0;
    for (int64_t k = lane; k < K; k += 32) m = fmax(m, fabs(src[r * kp + k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(~0u, m, o));
    if (lane == 0 && m > 0.0) atomic_max_pos(&rmax[r % R], m);
  }
}

// Column n of a B operand [P][K][N] whose N index is row-padded: n = y*w + c
// with c < wsrc real (source offset y*wsrc + c) and c >= wsrc zero.
__device__ __forceinline__ int64_t bsrc_col(int64_t n, int64_t w,
                                            int64_t wsrc) {
  const int64_t y = n / w, c = n - y * w;
  return c < wsrc ? y * wsrc + c : -1;
}

// cmax[n] = max over (p, k) |B[p][k][n]|; source rows of length ldsrc.
__global__ void colmax_kernel(const double *__restrict__ src, int64_t K,
                              int64_t N, int64_t w, int64_t wsrc,
                              int64_t ldsrc, unsigned long long *cmax) {
  const int64_t p = blockIdx.y;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = bsrc_col(n, w, wsrc);
    if (c < 0) continue;
    const double *s = src + p * K * ldsrc + c;
    double m = 0.0;
    for (int64_t k = 0; k < K; ++k) m = fmax(m, fabs(s[k * ldsrc]));
    if (m > 0.0) atomic_max_pos(&cmax[n], m);
  }
}

// e[x] = exponent with max(m1[x], m2[x] * s2) * 2^-e in [1/4, 1/2).
__global__ void exps_kernel(const unsigned long long *m1,
                            const unsigned long long *m2, double s2,
                            int64_t n, signed char *e) {
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n;
       x += (int64_t)gridDim.x * blockDim.x) {
    double m = __longlong_as_double((long long)m1[x]);
    if (m2) m = fmax(m, __longlong_as_double((long long)m2[x]) * s2);
    int E = 0;
    if (m > 0.0) frexp(m, &E);
    E += 1;
    e[x] = (signed char)(E < -120 ? -120 : E > 120 ? 120 : E);
  }
}

__device__ __forceinline__ void digits7(double s, int S, signed char *d) {
  for (int q = 0; q < S; ++q) {
    const double t = s * 128.0;
    const double r = rint(t);
    d[q] = (signed char)r;
    s = t - r;
  }
}

// s in (-1/2, 1/2): s = 2 sum_{q<S} d[q] 2^-8(q+1) + remainder.
__device__ __forceinline__ void digits8(double s, int S, signed char *d) {
  int v[8];
  double t = s * 128.0;
  double f = rint(t);
  v[0] = (int)f;
  s = t - f;                       // |s| <= 1/2
  for (int q = 1; q < S; ++q) {
    t = s * 256.0;
    f = rint(t);
    v[q] = (int)f;                 // in [-128, 128]
    s = t - f;
  }
  for (int q = S - 1; q >= 1; --q)
    if (v[q] == 128) {             // 128 * 2^-8q = -128 * 2^-8q + 2^-8(q-1)
      v[q] = -128;
      v[q - 1] += 1;
    }
  for (int q = 0; q < S; ++q) d[q] = (signed char)v[q];
}

// A side: src[npq][R][kp] (FP64) -> out[2S][npq][kpi/32][R][32] int8: digit
// planes of a * scale * 2^-ea[x], then their negatives.  Each 32-byte K
// chunk of R rows is contiguous, so a tensor-core tile's TMA box is one
// contiguous block of memory.
__global__ void slice_a_kernel(const double *__restrict__ src, int64_t npq,
                               int64_t R, int64_t K, int64_t kp, int64_t kpi,
                               double scale, const signed char *ea, int S,
                               int bits, signed char *__restrict__ out) {
  const int64_t n = npq * R * kpi, plane = n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t rr = i / kpi, k = i - rr * kpi;
    const int64_t pq = rr / R, r = rr - pq * R;
    const double a = k < K ? src[rr * kp + k] : 0.0;
    const double x = ldexp(a * scale, -ea[r]);
    signed char d[8], nd[8];
    if (bits == 8) {
      digits8(x, S, d);
      digits8(-x, S, nd);   // -(-128) does not fit a signed byte
    } else {
      digits7(x, S, d);
      for (int q = 0; q < S; ++q) nd[q] = (signed char)(-d[q]);
    }
    const int64_t o = pq * R * kpi + ((k / I8_KCHUNK) * R + r) * I8_KCHUNK +
                      (k % I8_KCHUNK);
    for (int q = 0; q < S; ++q) {
      out[q * plane + o] = d[q];
      out[(S + q) * plane + o] = nd[q];
    }
  }
}

// B side, transposed: B[P][K][N] (row-padded N, see bsrc_col) ->
// out[S][P][kpi/32][N][32] int8 digit planes of b * scale * 2^-eb[n]
// (32-byte K chunks of N columns contiguous).
__global__ void slice_b_kernel(const double *__restrict__ src, int K,
                               int64_t N, int64_t w, int64_t wsrc,
                               int64_t ldsrc, int64_t kpi, double scale,
                               const signed char *eb, int S, int bits,
                               int64_t P, signed char *__restrict__ out) {
  __shared__ double t[32][33];
  const int64_t p = blockIdx.z;
  const int64_t n0 = (int64_t)blockIdx.x * 32;
  const int k0 = blockIdx.y * 32;
  const double *s = src + p * K * ldsrc;
  for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
    const int k = k0 + rr;
    const int64_t n = n0 + threadIdx.x;
    const int64_t c = n < N ? bsrc_col(n, w, wsrc) : -1;
    t[rr][threadIdx.x] = (k < K && c >= 0) ? s[(int64_t)k * ldsrc + c] : 0.0;
  }
  __syncthreads();
  const int64_t plane = P * N * kpi;
  for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
    const int64_t n = n0 + rr;
    const int k = k0 + threadIdx.x;
    if (n < N && k < kpi) {
      signed char d[8];
      const double x = ldexp(t[threadIdx.x][rr] * scale, -eb[n]);
      if (bits == 8)
        digits8(x, S, d);
      else
        digits7(x, S, d);
      const int64_t o = p * N * kpi + ((int64_t)(k / I8_KCHUNK) * N + n) *
                                          I8_KCHUNK + (k % I8_KCHUNK);
      for (int q = 0; q < S; ++q) out[q * plane + o] = d[q];
    }
  }
}

int grid2(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t rowmax_launch(const double *src, int64_t npq, int64_t R, int64_t K,
                          int64_t kp, unsigned long long *rmax,
                          cudaStream_t st) {
  if (npq * R <= 0 || K <= 0) return cudaSuccess;
  rowmax_kernel<<<grid2(npq * R * 32), 256, 0, st>>>(src, npq, R, K, kp, rmax);
  return cudaGetLastError();
}

cudaError_t colmax_launch(const double *src, int64_t P, int64_t K, int64_t N,
                          int64_t w, int64_t wsrc, int64_t ldsrc,
                          unsigned long long *cmax, cudaStream_t st) {
  if (P <= 0 || K <= 0 || N <= 0) return cudaSuccess;
  for (int64_t p0 = 0; p0 < P; p0 += 65535) {
    const int64_t np_ = P - p0 < 65535 ? P - p0 : 65535;
    dim3 grid((unsigned)((N + 255) / 256 < 1024 ? (N + 255) / 256 : 1024),
              (unsigned)np_);
    colmax_kernel<<<grid, 256, 0, st>>>(src + p0 * K * ldsrc, K, N, w, wsrc,
                                        ldsrc, cmax);
  }
  return cudaGetLastError();
}

cudaError_t exps_launch(const unsigned long long *m1,
                        const unsigned long long *m2, double s2, int64_t n,
                        signed char *e, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  exps_kernel<<<grid2(n), 256, 0, st>>>(m1, m2, s2, n, e);
  return cudaGetLastError();
}

cudaError_t slice_a_launch(const double *src, int64_t npq, int64_t R,
                           int64_t K, int64_t kp, int64_t kpi, double scale,
                           const signed char *ea, int S, int bits,
                           signed char *out, cudaStream_t st) {
  if (npq * R <= 0) return cudaSuccess;
  if (bits != 7 && bits != 8) return cudaErrorInvalidValue;
  slice_a_kernel<<<grid2(npq * R * kpi), 256, 0, st>>>(src, npq, R, K, kp, kpi,
                                                       scale, ea, S, bits, out);
  return cudaGetLastError();
}

cudaError_t slice_b_launch(const double *src, int64_t P, int K, int64_t N,
                           int64_t w, int64_t wsrc, int64_t ldsrc, int64_t kpi,
                           double scale, const signed char *eb, int S,
                           int bits, signed char *out, cudaStream_t st) {
  if (P <= 0 || N <= 0 || kpi <= 0) return cudaSuccess;
  if (bits != 7 && bits != 8) return cudaErrorInvalidValue;
  for (int64_t p0 = 0; p0 < P; p0 += 65535) {
    const int64_t np_ = P - p0 < 65535 ? P - p0 : 65535;
    dim3 grid((unsigned)((N + 31) / 32), (unsigned)((kpi + 31) / 32),
              (unsigned)np_);
    // planes keep their full [P] extent: offset the output by p0 rows
    slice_b_kernel<<<grid, dim3(32, 8), 0, st>>>(
        src + p0 * K * ldsrc, K, N, w, wsrc, ldsrc, kpi, scale, eb, S, bits,
        P, out + p0 * N * kpi);
  }
  return cudaGetLastError();
}

}  // namespace ptb
