// Tensor-map views of the engine's operands: DMMA views of padded FP64
// blocks, TF32 plane views and their planes, INT8 digit-plane views.
// Part of the triples engine (plan_*.cu); internal declarations shared by
// those files are in plan_impl.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "plan_impl.h"

namespace ptb {

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType,
                                  cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p,
                                cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// A-view of a padded block [P][Q][R][Kpad] with logical K: dims (K, R, Q, P),
// box (4, bm, 1, 1).
int map_a(CUtensorMap *m, const double *p, int64_t K, int64_t R, int64_t Q,
          int64_t P, int bm) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  const int64_t kp = pad4(K);
  cuuint64_t dims[4] = {(cuuint64_t)std::max<int64_t>(K, 1),
                        (cuuint64_t)std::max<int64_t>(R, 1),
                        (cuuint64_t)std::max<int64_t>(Q, 1),
                        (cuuint64_t)std::max<int64_t>(P, 1)};
  cuuint64_t strides[3] = {(cuuint64_t)(kp * 8), (cuuint64_t)(R * kp * 8),
                           (cuuint64_t)(Q * R * kp * 8)};
  cuuint32_t box[4] = {4, (cuuint32_t)bm, 1, 1};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)p, dims,
                   strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (A view) failed: " + std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

// B-view of a padded block [P][K][Nld] with logical N: dims (N, K, P),
// box (4, GEMM_BK, 1).
int map_b(CUtensorMap *m, const double *p, int64_t N, int64_t Nld, int64_t K,
          int64_t P) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  cuuint64_t dims[3] = {(cuuint64_t)std::max<int64_t>(N, 1),
                        (cuuint64_t)std::max<int64_t>(K, 1),
                        (cuuint64_t)std::max<int64_t>(P, 1)};
  cuuint64_t strides[2] = {(cuuint64_t)(Nld * 8), (cuuint64_t)(K * Nld * 8)};
  cuuint32_t box[3] = {4, (cuuint32_t)GEMM_BK, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)p, dims,
                   strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (B view) failed: " + std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

int tc_encode(CUtensorMap *m, const float *p, int rank, const cuuint64_t *dims,
              const cuuint64_t *strides, const cuuint32_t *box) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, (void *)p, dims,
                   strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (tensor-core view) failed: " +
              std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

// Digit-plane views (see slice_a / slice_b): 32-byte K chunks of rows
// stored contiguously, boxes of 32 bytes x 128 (A) or bn (B) rows swizzled
// to 32 bytes.  A: (32, R, nK, Q*P, 2S); B: (32, N, nK, P, S).
int i8_map_a(CUtensorMap *m, const signed char *p, int64_t K, int64_t R,
             int64_t Q, int64_t P, int S) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  constexpr int W = I8_KCHUNK;
  const int64_t kpi = i8_kpad(K), nk = kpi / W, npq = Q * P;
  cuuint64_t dims[5] = {W, (cuuint64_t)R, (cuuint64_t)nk, (cuuint64_t)npq,
                        (cuuint64_t)(2 * S)};
  cuuint64_t str[4] = {W, (cuuint64_t)(R * W), (cuuint64_t)(R * kpi),
                       (cuuint64_t)(npq * R * kpi)};
  cuuint32_t box[5] = {W, (cuuint32_t)TC_BM, 1, 1, 1};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, (void *)p, dims, str,
                   box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (INT8 A view) failed: " +
              std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

int i8_map_b(CUtensorMap *m, const signed char *p, int64_t K, int64_t N,
             int64_t P, int S, int bn) {
  if (g_dry) return LIBPT_OK;   // sizing pass: no views needed
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return LIBPT_ERR_CUDA;
  }
  constexpr int W = I8_KCHUNK;
  const int64_t kpi = i8_kpad(K), nk = kpi / W;
  cuuint64_t dims[5] = {W, (cuuint64_t)N, (cuuint64_t)nk, (cuuint64_t)P,
                        (cuuint64_t)S};
  cuuint64_t str[4] = {W, (cuuint64_t)(N * W), (cuuint64_t)(N * kpi),
                       (cuuint64_t)(P * N * kpi)};
  cuuint32_t box[5] = {W, (cuuint32_t)bn, 1, 1, 1};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, (void *)p, dims, str,
                   box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (INT8 B view) failed: " +
              std::to_string(r));
    return LIBPT_ERR_CUDA;
  }
  return LIBPT_OK;
}

int dmma_map_a(CUtensorMap *m, const double *p, int64_t K, int64_t R,
               int64_t Q, int64_t P, int bm) {
  return map_a(m, p, K, R, Q, P, bm);
}

int dmma_map_b(CUtensorMap *m, const double *p, int64_t N, int64_t Nld,
               int64_t K, int64_t P) {
  return map_b(m, p, N, Nld, K, P);
}

int tc_map_a(CUtensorMap *m, const float *p, int64_t K, int64_t R, int64_t Q,
             int64_t P) {
  const int64_t kp = pad4(K);
  cuuint64_t dims[4] = {(cuuint64_t)std::max<int64_t>(K, 1),
                        (cuuint64_t)std::max<int64_t>(R, 1),
                        (cuuint64_t)std::max<int64_t>(Q, 1),
                        (cuuint64_t)std::max<int64_t>(P, 1)};
  cuuint64_t strides[3] = {(cuuint64_t)(kp * 4), (cuuint64_t)(R * kp * 4),
                           (cuuint64_t)(Q * R * kp * 4)};
  cuuint32_t box[4] = {(cuuint32_t)tc_kchunk_elems(TC_TF32), (cuuint32_t)TC_BM,
                       1, 1};
  return tc_encode(m, p, 4, dims, strides, box);
}

int tc_map_b(CUtensorMap *m, const float *p, int64_t K, int64_t N, int64_t P) {
  const int64_t kp = pad4(K);
  cuuint64_t dims[3] = {(cuuint64_t)std::max<int64_t>(K, 1),
                        (cuuint64_t)std::max<int64_t>(N, 1),
                        (cuuint64_t)std::max<int64_t>(P, 1)};
  cuuint64_t strides[2] = {(cuuint64_t)(kp * 4), (cuuint64_t)(N * kp * 4)};
  cuuint32_t box[3] = {(cuuint32_t)tc_kchunk_elems(TC_TF32), (cuuint32_t)TC_BN,
                       1};
  return tc_encode(m, p, 3, dims, strides, box);
}

// TF32 planes of an operand, made once per (source block, role).
int get_planes(libpt_plan *p, const OpDesc &d, Planes *out) {
  const std::pair<const double *, int> key(d.src, d.role);
  for (auto &e : p->planes)
    if (e.first == key) {
      *out = e.second;
      return LIBPT_OK;
    }
  Planes pl;
  const int64_t kp = pad4(d.K);
  if (d.role == 0) {
    const int64_t n = d.P * d.Q * d.R * kp;
    if (dalloc(p, (void **)&pl.hi, n * 4) || dalloc(p, (void **)&pl.lo, n * 4))
      return LIBPT_ERR_NOMEM;
    DEV(split_tf32_launch(d.src, pl.hi, pl.lo, n, p->st));
  } else {
    const int64_t n = d.P * d.N * kp;
    if (dalloc(p, (void **)&pl.hi, n * 4) || dalloc(p, (void **)&pl.lo, n * 4))
      return LIBPT_ERR_NOMEM;
    DEV(transpose_split_tf32_launch(d.src, pl.hi, pl.lo, d.P, (int)d.K, d.N,
                                   d.Nld, kp, p->st));
  }
  p->planes.push_back({key, pl});
  *out = pl;
  return LIBPT_OK;
}

// Tensor-core views of a case: plane pairs at map indices 2i, 2i+1.
int build_tc(libpt_plan *p, SpinCase &c) {
  for (int i = 0; i < MAX_MAPS; ++i) {
    const OpDesc &d = c.opd[i];
    if (d.role < 0) continue;
    if (2 * i + 1 >= TC_MAX_MAPS) {
      set_error("too many tensor-core operand views");
      return LIBPT_ERR_ARG;
    }
    Planes pl;
    if (int r = get_planes(p, d, &pl)) return r;
    for (int h = 0; h < 2; ++h) {
      const float *pp = h ? pl.lo : pl.hi;
      int r = d.role == 0 ? tc_map_a(&c.tcmaps.m[2 * i + h], pp, d.K, d.R, d.Q, d.P)
                          : tc_map_b(&c.tcmaps.m[2 * i + h], pp, d.K, d.N, d.P);
      if (r) return r;
    }
  }
  return LIBPT_OK;
}

}  // namespace ptb
