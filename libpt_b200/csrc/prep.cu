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
