// Upstream producer on the device: the restricted (T) inputs of pt.h built
// where a density-fitted closed-shell CCSD leaves its results, so that a
// caller whose CCSD ran on the GPU hands libpt_rpt_dev (or a plan) device
// arrays without assembling the 74 GB of o=45, v=477 integrals on the host.
//
// From three-index factors B[Q][p][q] (naux auxiliary functions, row-major)
// of the occupied-occupied, occupied-virtual and virtual-virtual pairs, the
// abab blocks are Mulliken products
//     i_oovv[i][j][a][b] = (ia|jb) = sum_Q B_ov[Q][i][a] B_ov[Q][j][b]
//     i_ovvv[i][a][b][c] = (ib|ac) = sum_Q B_ov[Q][i][b] B_vv[Q][a][c]
//     i_oovo[i][j][a][k] = (ia|jk) = sum_Q B_ov[Q][i][a] B_oo[Q][j][k]
// and the same-spin blocks their antisymmetrised forms
//     oovv aaaa = abab - abab(a <-> b),  oovo aaaa = abab - abab(i <-> j),
//     ovvv aaaa = abab - abab(b <-> c) packed over b > c (pair b(b-1)/2 + c),
//     t2 aaaa   = t2 abab - t2 abab(a <-> b).
// These are the relations the reference's own restricted fixtures satisfy
// (tests/golden rpt02/rpt09: abab blocks with the (ia|jb), (ib|ac), (ia|jk)
// index symmetries, aaaa blocks = abab minus its swap; checked on the CPU in
// tests/test_producer.py); pt.h documents only "properly (anti-)symmetrized"
// (src/pt.h:37-57).  No counterpart in the reference: its caller (Q-Chem,
// README.md:5-6) builds these arrays itself.
//
// Each product is one plain FP64 GEMM, done by cuBLAS (loaded at the first
// call with dlopen, so the library itself keeps no link-time dependency on
// it); the GEMM writes its result in the order of its operands, and this
// file's kernels move it into the pt.h order and form the same-spin blocks:
// row copies with a permuted row index (each row a contiguous run of the
// last pt.h index, read and written coalesced) and a 32 x 32 shared-memory
// tile transpose for the antisymmetrisations.  The oovv and oovo products
// are first written into the same-spin half of their output arrays, which
// holds exactly as many elements, so no scratch is needed there; the OVVV
// product goes through one v^3 scratch block per occupied index
// (stream-ordered allocation).  Cost: 2 o v naux (o v + o^2 + v^2) flops,
// 1.7e13 at o=45, v=477, naux=1566 (the OVVV term 2 o v^3 naux 1.5e13),
// against 2.3e16 for the (T) solve of those inputs.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <climits>
#include <mutex>
#include <string>

#include "plan.h"
#include "pt.h"

#define LIBPT_API extern "C" __attribute__((visibility("default")))

namespace {

// ---- cuBLAS, resolved at run time -------------------------------------------
struct Blas {
  bool ok = false;
  std::string why;
  decltype(&cublasCreate_v2) create = nullptr;
  decltype(&cublasDestroy_v2) destroy = nullptr;
  decltype(&cublasSetStream_v2) set_stream = nullptr;
  decltype(&cublasDgemm_v2) dgemm = nullptr;
};

Blas &blas() {
  static Blas b;
  static std::once_flag once;
  std::call_once(once, [] {
    void *h = dlopen("libcublas.so.12", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
      b.why = std::string("cannot load libcublas.so.12: ") + dlerror();
      return;
    }
    b.create = reinterpret_cast<decltype(b.create)>(dlsym(h, "cublasCreate_v2"));
    b.destroy =
        reinterpret_cast<decltype(b.destroy)>(dlsym(h, "cublasDestroy_v2"));
    b.set_stream =
        reinterpret_cast<decltype(b.set_stream)>(dlsym(h, "cublasSetStream_v2"));
    b.dgemm = reinterpret_cast<decltype(b.dgemm)>(dlsym(h, "cublasDgemm_v2"));
    b.ok = b.create && b.destroy && b.set_stream && b.dgemm;
    if (!b.ok) b.why = "libcublas.so.12 lacks a needed entry point";
  });
  return b;
}

// ---- layout kernels -------------------------------------------------------------

// dst row r = (x, y, z) of an n0 x n1 x n2 row grid (z fastest) is the
// source row at x s0 + y s1 + z s2; rows of L elements, one warp per row.
__global__ void rows3_kernel(double *__restrict__ dst,
                             const double *__restrict__ src, int64_t n0,
                             int64_t n1, int64_t n2, int64_t L, int64_t s0,
                             int64_t s1, int64_t s2) {
  const int64_t nrows = n0 * n1 * n2;
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       r < nrows; r += warps) {
    const int64_t z = r % n2, y = (r / n2) % n1, x = r / (n1 * n2);
    const double *s = src + x * s0 + y * s1 + z * s2;
    double *d = dst + r * L;
    for (int64_t e = lane; e < L; e += 32) d[e] = s[e];
  }
}

// For each of nblk n x n blocks, block blk of the source at
// (blk / nj) si + (blk % nj) sj with rows ld apart:
//   dense:  dst[blk][x][y] = src[blk][x][y] - src[blk][y][x]
//   packed: dst[blk][x(x-1)/2 + y] = the same, for x > y (block stride
//           n(n-1)/2 in dst)
// A CTA handles a 32 x 32 tile (blockIdx.x) of block blk0 + blockIdx.y: the
// mirrored tile is staged through shared memory so both reads are coalesced.
__global__ void antisym_kernel(double *__restrict__ dst,
                               const double *__restrict__ src, int n,
                               bool packed, int64_t blk0, int64_t ld,
                               int64_t nj, int64_t si, int64_t sj) {
  __shared__ double t[32][33];
  const int nt = (n + 31) / 32;
  const int x0 = (blockIdx.x / nt) * 32, y0 = (blockIdx.x % nt) * 32;
  if (packed && x0 + 31 <= y0) return;   // no x > y in this tile
  const int64_t blk = blk0 + blockIdx.y;
  const double *s = src + (blk / nj) * si + (blk % nj) * sj;
  const int lx = threadIdx.x, ly = threadIdx.y;   // 32 x 8 threads
  // t[y - y0][x - x0] = src[y][x] for the mirrored tile (rows y0.., cols x0..)
  for (int r = ly; r < 32; r += 8) {
    const int y = y0 + r, x = x0 + lx;
    t[r][lx] = (y < n && x < n) ? s[(int64_t)y * ld + x] : 0.0;
  }
  __syncthreads();
  for (int r = ly; r < 32; r += 8) {
    const int x = x0 + r, y = y0 + lx;
    if (x >= n || y >= n) continue;
    const double v = s[(int64_t)x * ld + y] - t[lx][r];
    if (!packed)
      dst[blk * (int64_t)n * n + (int64_t)x * n + y] = v;
    else if (x > y)
      dst[blk * ((int64_t)n * (n - 1) / 2) + (int64_t)x * (x - 1) / 2 + y] = v;
  }
}

// Same-spin OOVO from its GEMM result Y[(i,a)][(j,k)] = (ia|jk):
// dst[i][j][a][k] = Y[(i v + a) o^2 + j o + k] - Y[(j v + a) o^2 + i o + k]
// (both reads contiguous in k).
__global__ void oovo_same_kernel(double *__restrict__ dst,
                                 const double *__restrict__ y, int64_t o,
                                 int64_t v) {
  const int64_t total = o * o * v * o;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e % o, a = (e / o) % v, j = (e / (o * v)) % o,
                  i = e / (o * v * o);
    dst[e] = y[(i * v + a) * o * o + j * o + k] -
             y[(j * v + a) * o * o + i * o + k];
  }
}

// dst[i][j][e] = src[i][j][e] - src[j][i][e] for i, j < o, e < m.
__global__ void swap_sub_kernel(double *__restrict__ dst,
                                const double *__restrict__ src, int64_t o,
                                int64_t m) {
  const int64_t total = o * o * m;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % m, ij = e / m, i = ij / o, j = ij % o;
    dst[e] = src[e] - src[(j * o + i) * m + r];
  }
}

int rows3(double *dst, const double *src, int64_t n0, int64_t n1, int64_t n2,
          int64_t L, int64_t s0, int64_t s1, int64_t s2, cudaStream_t st) {
  const int64_t nrows = n0 * n1 * n2;
  if (nrows == 0 || L == 0) return LIBPT_OK;
  const int grid = (int)std::min<int64_t>((nrows + 7) / 8, 148 * 32);
  rows3_kernel<<<grid, 256, 0, st>>>(dst, src, n0, n1, n2, L, s0, s1, s2);
  CK(cudaGetLastError());
  return LIBPT_OK;
}

// antisym_kernel over nblk blocks (see there); contiguous n x n blocks by
// default.
int antisym(double *dst, const double *src, int64_t nblk, int n, bool packed,
            cudaStream_t st, int64_t ld = -1, int64_t nj = 1, int64_t si = -1,
            int64_t sj = 0) {
  if (nblk <= 0 || n <= 0) return LIBPT_OK;
  if (ld < 0) ld = n;
  if (si < 0) si = (int64_t)n * n;
  const int nt = (n + 31) / 32;
  for (int64_t b0 = 0; b0 < nblk; b0 += 65535) {   // grid.y limit
    const int64_t nb = std::min<int64_t>(nblk - b0, 65535);
    antisym_kernel<<<dim3(nt * nt, (unsigned)nb), dim3(32, 8), 0, st>>>(
        dst, src, n, packed, b0, ld, nj, si, sj);
    CK(cudaGetLastError());
  }
  return LIBPT_OK;
}

int oovo_same(double *dst, const double *y, int64_t o, int64_t v,
              cudaStream_t st) {
  const int64_t total = o * o * v * o;
  if (total == 0) return LIBPT_OK;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  oovo_same_kernel<<<grid, 256, 0, st>>>(dst, y, o, v);
  CK(cudaGetLastError());
  return LIBPT_OK;
}

int swap_sub(double *dst, const double *src, int64_t o, int64_t m,
             cudaStream_t st) {
  const int64_t total = o * o * m;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  swap_sub_kernel<<<grid, 256, 0, st>>>(dst, src, o, m);
  CK(cudaGetLastError());
  return LIBPT_OK;
}

// C (column-major m x n, ldc) = A (m x k, lda) * B^T (B: n x k, ldb)
int gemm_nt(cublasHandle_t h, int m, int n, int k, const double *A, int lda,
            const double *B, int ldb, double *C, int ldc) {
  if (m == 0 || n == 0) return LIBPT_OK;   // an empty spin block
  const double one = 1.0, zero = 0.0;
  const cublasStatus_t s = blas().dgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, m, n, k,
                                        &one, A, lda, B, ldb, &zero, C, ldc);
  if (s != CUBLAS_STATUS_SUCCESS) {
    ptb::set_error("cublasDgemm: status " + std::to_string((int)s));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

int produce(size_t o_, size_t v_, size_t naux_, const double *b_oo,
            const double *b_ov, const double *b_vv, const double *t2_abab,
            double *t2, double *i_oovo, double *i_oovv, double *i_ovvv,
            cudaStream_t st, cublasHandle_t h) {
  const int64_t o = (int64_t)o_, v = (int64_t)v_, q = (int64_t)naux_;
  const int64_t ov = o * v, oovv = o * o * v * v, oovo = o * o * v * o;
  const int64_t npair = v * (v - 1) / 2;
  // amplitudes: abab as given, aaaa its antisymmetrised form
  if (t2_abab) {
    if (t2_abab != t2 + oovv)
      CK(cudaMemcpyAsync(t2 + oovv, t2_abab, (size_t)oovv * sizeof(double),
                         cudaMemcpyDeviceToDevice, st));
    if (int r = antisym(t2, t2 + oovv, o * o, (int)v, false, st)) return r;
  }
  // OOVV: W[(i,a)][(j,b)] into the aaaa half, then abab, then aaaa
  if (int r = gemm_nt(h, (int)ov, (int)ov, (int)q, b_ov, (int)ov, b_ov,
                      (int)ov, i_oovv, (int)ov))
    return r;
  if (int r = rows3(i_oovv + oovv, i_oovv, o, o, v, v, v * ov, v, ov, st))
    return r;
  if (int r = antisym(i_oovv, i_oovv + oovv, o * o, (int)v, false, st))
    return r;
  // OOVO: Y[(i,a)][(j,k)] into the aaaa half, then abab, then aaaa
  if (int r = gemm_nt(h, (int)(o * o), (int)ov, (int)q, b_oo, (int)(o * o),
                      b_ov, (int)ov, i_oovo, (int)(o * o)))
    return r;
  if (int r = rows3(i_oovo + oovo, i_oovo, o, o, v, o, v * o * o, o, o * o, st))
    return r;
  if (int r = swap_sub(i_oovo, i_oovo + oovo, o, v * o, st)) return r;
  // OVVV, one occupied index at a time: Z[b][(a,c)] (v^3 scratch), then the
  // abab slice [a][b][c], then its packed aaaa slice
  double *z = nullptr;
  CK(cudaMallocAsync((void **)&z, (size_t)(v * v * v) * sizeof(double), st));
  int r = LIBPT_OK;
  double *ovvv_ab = i_ovvv + o * v * npair;
  for (int64_t i = 0; i < o && !r; ++i) {
    r = gemm_nt(h, (int)(v * v), (int)v, (int)q, b_vv, (int)(v * v),
                b_ov + i * v, (int)ov, z, (int)(v * v));
    if (!r) r = rows3(ovvv_ab + i * v * v * v, z, 1, v, v, v, 0, v, v * v, st);
    if (!r)
      r = antisym(i_ovvv + i * v * npair, ovvv_ab + i * v * v * v, v, (int)v,
                  true, st);
  }
  cudaError_t e = cudaFreeAsync(z, st);
  if (!r && e != cudaSuccess) {
    ptb::set_error(std::string("cudaFreeAsync: ") + cudaGetErrorString(e));
    r = LIBPT_ERR_CUDA;
  }
  return r;
}

// Unrestricted: factors of each spin (alpha a, beta b); the pt.h blocks
// aaaa / abab / bbbb / baba of each family (src/pt.h:64-100 sizes):
//   oovv abab[i a][j b][a a][b b] = (ia|jb) = sum_Q Ba_ov[i][a] Bb_ov[j][b]
//   oovo abab[i a][j b][a a][k b] = (ia|jk) = sum_Q Ba_ov[i][a] Bb_oo[j][k]
//   ovvv abab[i a][a b][b a][c b] = (ib|ac) = sum_Q Ba_ov[i][b] Bb_vv[a][c]
// baba the same with the spins exchanged, aaaa / bbbb the antisymmetrised
// same-spin products of one spin's factors (formed straight from the GEMM
// results, whose mirrored elements the tile transpose reads).
struct Spin {
  int64_t o, v;
  const double *oo, *ov, *vv;
};

int same_spin(const Spin &x, double *oovo_aa, double *oovv_aa,
              double *ovvv_aa, double *scr, cudaStream_t st, cublasHandle_t h,
              int64_t q) {
  const int64_t o = x.o, v = x.v, ov = o * v, npair = v * (v - 1) / 2;
  if (o == 0 || v == 0) return LIBPT_OK;
  // OOVV: W[(i,a)][(j,b)]; aaaa[i][j][a][b] = W[ia][jb] - W[ib][ja]
  if (int r = gemm_nt(h, (int)ov, (int)ov, (int)q, x.ov, (int)ov, x.ov,
                      (int)ov, scr, (int)ov))
    return r;
  if (int r = antisym(oovv_aa, scr, o * o, (int)v, false, st, ov, o, v * ov, v))
    return r;
  // OOVO: Y[(i,a)][(j,k)]
  if (int r = gemm_nt(h, (int)(o * o), (int)ov, (int)q, x.oo, (int)(o * o),
                      x.ov, (int)ov, scr, (int)(o * o)))
    return r;
  if (int r = oovo_same(oovo_aa, scr, o, v, st)) return r;
  // OVVV per occupied index: Z[b][(a,c)]; packed aaaa[a][b > c] =
  // Z[b][a][c] - Z[c][a][b]
  for (int64_t i = 0; i < o; ++i) {
    if (int r = gemm_nt(h, (int)(v * v), (int)v, (int)q, x.vv, (int)(v * v),
                        x.ov + i * v, (int)ov, scr, (int)(v * v)))
      return r;
    if (int r = antisym(ovvv_aa + i * v * npair, scr, v, (int)v, true, st,
                        v * v, 1, v, 0))
      return r;
  }
  return LIBPT_OK;
}

// The mixed-spin blocks with occupied / first virtual index of spin x and
// the others of spin y (abab for x = alpha, baba for x = beta).
int mixed_spin(const Spin &x, const Spin &y, double *oovo_xy, double *oovv_xy,
               double *ovvv_xy, double *scr, cudaStream_t st,
               cublasHandle_t h, int64_t q) {
  const int64_t ox = x.o, vx = x.v, oy = y.o, vy = y.v;
  const int64_t oxvx = ox * vx, oyvy = oy * vy;
  if (ox == 0 || vx == 0) return LIBPT_OK;
  // OOVV [i x][j y][a x][b y]: W[(i,a)][(j,b)]
  if (oy > 0 && vy > 0) {
    if (int r = gemm_nt(h, (int)oyvy, (int)oxvx, (int)q, y.ov, (int)oyvy,
                        x.ov, (int)oxvx, scr, (int)oyvy))
      return r;
    if (int r = rows3(oovv_xy, scr, ox, oy, vx, vy, vx * oyvy, vy, oyvy, st))
      return r;
  }
  // OOVO [i x][j y][a x][k y]: Y[(i,a)][(j,k)]
  if (oy > 0) {
    if (int r = gemm_nt(h, (int)(oy * oy), (int)oxvx, (int)q, y.oo,
                        (int)(oy * oy), x.ov, (int)oxvx, scr, (int)(oy * oy)))
      return r;
    if (int r = rows3(oovo_xy, scr, ox, oy, vx, oy, vx * oy * oy, oy, oy * oy,
                      st))
      return r;
  }
  // OVVV [i x][a y][b x][c y] per i: Z[b][(a,c)]
  if (vy > 0)
    for (int64_t i = 0; i < ox; ++i) {
      if (int r = gemm_nt(h, (int)(vy * vy), (int)vx, (int)q, y.vv,
                          (int)(vy * vy), x.ov + i * vx, (int)oxvx, scr,
                          (int)(vy * vy)))
        return r;
      if (int r = rows3(ovvv_xy + i * vy * vx * vy, scr, 1, vy, vx, vy, 0, vy,
                        vy * vy, st))
        return r;
    }
  return LIBPT_OK;
}

int produce_u(const Spin &A, const Spin &B, double *i_oovo, double *i_oovv,
              double *i_ovvv, cudaStream_t st, cublasHandle_t h, int64_t q) {
  const int64_t oa = A.o, va = A.v, ob = B.o, vb = B.v;
  const int64_t npa = va * (va - 1) / 2, npb = vb * (vb - 1) / 2;
  // block offsets (aaaa, abab, bbbb, baba) of each family
  const int64_t vv0 = oa * oa * va * va, vv1 = vv0 + oa * ob * va * vb,
                vv2 = vv1 + ob * ob * vb * vb;
  const int64_t vo0 = oa * oa * va * oa, vo1 = vo0 + oa * ob * va * ob,
                vo2 = vo1 + ob * ob * vb * ob;
  const int64_t v30 = oa * va * npa, v31 = v30 + oa * vb * va * vb,
                v32 = v31 + ob * vb * npb;
  // scratch: the largest GEMM result
  int64_t need = std::max<int64_t>({oa * va * oa * va, ob * vb * ob * vb,
                                    oa * va * ob * vb, oa * va * oa * oa,
                                    ob * vb * ob * ob, oa * va * ob * ob,
                                    ob * vb * oa * oa, va * va * va,
                                    vb * vb * vb, va * vb * vb, vb * va * va,
                                    1});
  double *scr = nullptr;
  CK(cudaMallocAsync((void **)&scr, (size_t)need * sizeof(double), st));
  int r = same_spin(A, i_oovo, i_oovv, i_ovvv, scr, st, h, q);
  if (!r) r = same_spin(B, i_oovo + vo1, i_oovv + vv1, i_ovvv + v31, scr, st,
                        h, q);
  if (!r) r = mixed_spin(A, B, i_oovo + vo0, i_oovv + vv0, i_ovvv + v30, scr,
                         st, h, q);
  if (!r) r = mixed_spin(B, A, i_oovo + vo2, i_oovv + vv2, i_ovvv + v32, scr,
                         st, h, q);
  cudaError_t e = cudaFreeAsync(scr, st);
  if (!r && e != cudaSuccess) {
    ptb::set_error(std::string("cudaFreeAsync: ") + cudaGetErrorString(e));
    r = LIBPT_ERR_CUDA;
  }
  return r;
}

// cuBLAS handle on `stream` around f(handle); status of f or of the set-up.
template <typename F>
int with_blas(const char *who, void *stream, F f) {
  Blas &b = blas();
  if (!b.ok) {
    ptb::set_error(std::string(who) + ": " + b.why);
    return LIBPT_ERR_CUDA;
  }
  cublasHandle_t h = nullptr;
  if (b.create(&h) != CUBLAS_STATUS_SUCCESS) {
    ptb::set_error(std::string(who) + ": cublasCreate failed");
    return LIBPT_ERR_CUDA;
  }
  int r = b.set_stream(h, static_cast<cudaStream_t>(stream)) ==
                  CUBLAS_STATUS_SUCCESS
              ? LIBPT_OK
              : LIBPT_ERR_CUDA;
  if (r) ptb::set_error(std::string(who) + ": cublasSetStream failed");
  if (!r) r = f(h);
  b.destroy(h);
  return r;
}

}  // namespace

LIBPT_API int libpt_rpt_inputs_df(size_t o, size_t v, size_t naux,
                                  const double *b_oo, const double *b_ov,
                                  const double *b_vv, const double *t2_abab,
                                  double *t2, double *i_oovo, double *i_oovv,
                                  double *i_ovvv, void *stream) {
  if (o == 0 || v == 0 || naux == 0 || !b_oo || !b_ov || !b_vv || !i_oovo ||
      !i_oovv || !i_ovvv || (t2_abab && !t2)) {
    ptb::set_error("libpt_rpt_inputs_df: zero size or NULL array");
    return LIBPT_ERR_ARG;
  }
  // cuBLAS takes int dimensions: o v, o^2, v^2 and naux must fit
  const size_t lim = (size_t)INT_MAX;
  if (o > lim / v || v > 46340 || o > 46340 || naux > lim) {
    ptb::set_error("libpt_rpt_inputs_df: sizes too large");
    return LIBPT_ERR_ARG;
  }
  return with_blas("libpt_rpt_inputs_df", stream, [&](cublasHandle_t h) {
    return produce(o, v, naux, b_oo, b_ov, b_vv, t2_abab, t2, i_oovo, i_oovv,
                   i_ovvv, static_cast<cudaStream_t>(stream), h);
  });
}

LIBPT_API int libpt_upt_inputs_df(
    size_t oa, size_t va, size_t ob, size_t vb, size_t naux,
    const double *b_oo_a, const double *b_ov_a, const double *b_vv_a,
    const double *b_oo_b, const double *b_ov_b, const double *b_vv_b,
    double *i_oovo, double *i_oovv, double *i_ovvv, void *stream) {
  // a factor array may be NULL only when it has no elements
  if (oa + ob == 0 || va + vb == 0 || naux == 0 || !i_oovo || !i_oovv ||
      !i_ovvv || (oa && !b_oo_a) || (oa && va && !b_ov_a) ||
      (va && !b_vv_a) || (ob && !b_oo_b) || (ob && vb && !b_ov_b) ||
      (vb && !b_vv_b)) {
    ptb::set_error("libpt_upt_inputs_df: zero size or NULL array");
    return LIBPT_ERR_ARG;
  }
  // cuBLAS takes int dimensions: o v, o^2 and v^2 of each spin must fit
  const size_t lim = (size_t)INT_MAX, big = std::max({oa, va, ob, vb});
  if (big > 46340 || naux > lim || oa * va > lim || ob * vb > lim) {
    ptb::set_error("libpt_upt_inputs_df: sizes too large");
    return LIBPT_ERR_ARG;
  }
  const Spin A{(int64_t)oa, (int64_t)va, b_oo_a, b_ov_a, b_vv_a};
  const Spin B{(int64_t)ob, (int64_t)vb, b_oo_b, b_ov_b, b_vv_b};
  return with_blas("libpt_upt_inputs_df", stream, [&](cublasHandle_t h) {
    return produce_u(A, B, i_oovo, i_oovv, i_ovvv,
                     static_cast<cudaStream_t>(stream), h, (int64_t)naux);
  });
}
