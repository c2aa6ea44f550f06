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
