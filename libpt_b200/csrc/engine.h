// Host/device shared structures of the triples engine.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ptb {

// ---- FP64 DMMA GEMM ------------------------------------------------------
//
// One "job" is C[M][N] = sum over segments s of (+/-) A_s B_s for one
// triple, where A_s is a [rows][K_s] slice of a padded amplitude/OOVO block
// (TMA view: dims (K, rows, Q, P)) and B_s a [K_s][N] slice of a padded
// OVVV/amplitude block (TMA view: dims (N, K, P)).  The slices are selected
// by the occupied indices (Q, P) resp. (P) of the triple.

constexpr int GEMM_BM = 128;   // rows of a CTA tile (96 or 128, per case)
constexpr int GEMM_BN = 128;   // columns of a CTA tile
constexpr int GEMM_BK = 16;    // contraction depth of one pipeline stage
constexpr int GEMM_STAGES = 5;
constexpr int GEMM_CONSUMER_WARPS = 8;
constexpr int GEMM_THREADS = (GEMM_CONSUMER_WARPS + 1) * 32;
constexpr int MAX_SEG = 6;
constexpr int MAX_MAPS = 24;

struct GemmSeg {
  int16_t amap, bmap;   // indices into MapSet
  int16_t neg, pad_;    // neg != 0: subtract this product
  int32_t a_q, a_p;     // A-view coordinates of dims 2 and 3
  int32_t b_p;          // B-view coordinate of dim 2
  int32_t ksteps;       // ceil(K_s / GEMM_BK)
};

struct GemmJob {
  double *out;          // C, row-major with leading dimension ldc
  int64_t ldc;
  int32_t M, N;         // N <= ldc, N % 4 == 0
  int32_t ntiles_n;     // ceil(N / GEMM_BN)
  int32_t tile_begin;   // first flat tile index of this job in the launch
  int32_t nseg;
  int32_t mtiles;       // ceil(M / BM); tiles are numbered M-tile fastest
  GemmSeg seg[MAX_SEG];
  // emulated FP64: power-of-two exponents of the output rows / columns
  const signed char *ea, *eb;
};

struct MapSet {
  CUtensorMap m[MAX_MAPS];
};

size_t gemm_smem_bytes(int bm);
// bm: CTA tile rows, 96 or 128 (the A views' box height must match).
cudaError_t gemm_dmma_launch(const MapSet &maps, const GemmJob *d_jobs,
                             int njobs, int total_tiles, int bm,
                             unsigned *d_err, cudaStream_t st);

// ---- tensor-core (tcgen05) GEMM --------------------------------------------
//
// Operands as "planes" (e.g. TF32 hi / lo parts).  A planes: [P][Q][R][Kp]
// (K contiguous) seen as (K, R, Q, P) with boxes (KCHUNK bytes, 128, 1, 1);
// B planes transposed, [P][N][Kp], seen as (K, N, P) with boxes
// (KCHUNK bytes, TC_BN, 1); both 128B-swizzled.  Plane p of an operand whose
// first plane is map i is map i + p.

constexpr int TC_BM = 128;    // rows of a tile (TMEM lanes)
constexpr int TC_BN = 256;    // columns of a tile
constexpr int TC_TF32 = 0;    // kinds
constexpr int TC_INT8 = 1;
constexpr int TC_S_MIN = 4, TC_S_MAX = 7;
constexpr int TC_MAX_MAPS = 48;

struct TcMapSet {
  CUtensorMap m[TC_MAX_MAPS];
};

struct TcProducts {           // acc[c] += A_plane[pa] * B_plane[pb]^T
  int8_t pa[16], pb[16], acc[16];
  int n;
};

int tc_kchunk_elems(int kind);   // K elements per pipeline stage (TF32)
// 3xTF32: planes {hi, lo} in separate maps (2i, 2i+1), products from prods.
cudaError_t gemm_tc_launch(int kind, const TcMapSet &maps,
                           const GemmJob *d_jobs, int njobs, int total_tiles,
                           const TcProducts &prods, unsigned *d_err,
                           cudaStream_t st, int slices = 0);

// ---- emulated FP64 (tcgen05 kind::i8, gemm_i8.cu) ---------------------------
//
// S digit planes per operand, the products with p + q <= S - 1 (0-based)
// into S INT32 accumulators of bn columns.  The digit planes are a
// coordinate of one map per operand: A maps [2S][P][Q][kpi/32][R][32] hold
// the digits then their negatives, B maps [S][P][kpi/32][N][32]; 32-byte K
// chunks of 128 (A) or bn (B) rows are contiguous, read as one TMA box each
// and swizzled to 32 bytes.  An A segment's (Q, P) coordinates are merged
// into a_q = a_p * Q + a_q.
struct I8Tile {
  int bn;   // tile columns (multiple of 16, S * bn <= 512)
  int kc;   // K bytes per pipeline stage (32 or 64: one or two MMA K steps)
};
// K padded to whole 32-byte chunks: the row extent of the digit planes.
inline int64_t i8_kpad(int64_t K) { return (K + 31) & ~int64_t(31); }
// The tile variants compiled for a slice count (widest first); returns
// their number (0 for an unsupported count).
int i8_tiles(int slices, const I8Tile **out);
cudaError_t gemm_i8_launch(int slices, I8Tile tile, const TcMapSet &maps,
                           const GemmJob *d_jobs, int njobs, int total_tiles,
                           unsigned *d_err, cudaStream_t st);

// ---- energy epilogues ------------------------------------------------------

constexpr int EPI_A = 8, EPI_B = 8, EPI_C = 32;   // tile extents a x b x c
constexpr int EPI_THREADS = 256;
constexpr int EPI_CS = EPI_C + 2;                 // smem row stride (banks)

// Arguments shared by the same-spin (aaa) and mixed-spin (aab) epilogues.
struct EpiArgs {
  const double *ws;       // triple t's arrays start at ws + t * ws_stride
  int64_t ws_stride;
  int64_t offL[3];        // array offsets of the (first) amplitude W / L
  int64_t offR[3];        // offsets of R for (fT); offR[0] < 0 for (T)
  int64_t ld[3];          // leading dims: aaa {ldT}; aab {ldU1, ldU2, ldP}
  int64_t rowU1, rowU2;   // aab: padded inner extents of U1 (vb) and U2 (va)
  const int *trip;        // i, j, k per triple of the batch
  int oa, va, ob, vb;
  const double *d_a, *d_b;                  // denominators [o][v]
  const double *ov1_a, *ov1_b;              // t1 / l1
  const double *g1_ab, *g1_aa;              // i_oovv blocks
  int64_t g1_ld_ab, g1_ld_aa;               // their inner leading dims
  const double *ov2_a, *ov2_b;              // f_ov / f2_ov
  const double *g2_ab, *g2_aa;              // t2 / l2 blocks
  int64_t g2_ld_ab, g2_ld_aa;
  double *partials;       // [ntrip][ntiles]
  int ntiles;
  const int4 *tiles;      // aaa: (a0, b0, c0); aab: (a0, b0, 0) block pairs
  int ctiles;             // aab: number of c blocks
};

size_t epi_smem_bytes(bool aab, bool ft);
cudaError_t epi_aaa_launch(const EpiArgs &a, bool ft, int ntrip,
                           cudaStream_t st);
cudaError_t epi_aab_launch(const EpiArgs &a, bool ft, int ntrip,
                           cudaStream_t st);
// e_slot[slot[t]] = fixed-order sum of partials[t][0..ntiles).
cudaError_t reduce_partials_launch(const double *partials, int ntiles,
                                   int ntrip, const int *slot, double *e_slot,
                                   cudaStream_t st);

// ---- operand preparation ---------------------------------------------------

// dst[r][c] = src[r][c] (c < w), 0 (w <= c < dpitch); converts FP32 to FP64.
cudaError_t repack_launch(const void *src, bool src_fp32, double *dst,
                          int64_t rows, int64_t w, int64_t dpitch,
                          cudaStream_t st);
// out[p][q][pair(a,b)] = tau[p][q][a][b] for a > b (pair = a(a-1)/2 + b);
// tau rows padded to ldv, out rows padded to ldp (zero fill).
cudaError_t pack_pairs_launch(const double *tau, double *out, int64_t npq,
                              int v, int64_t ldv, int64_t ldp,
                              cudaStream_t st);
// TF32 hi/lo planes of n FP64 values (exact FP32 values).
cudaError_t split_tf32_launch(const double *src, float *hi, float *lo,
                              int64_t n, cudaStream_t st);
// src[P][K][ldn] -> hi/lo[P][N][ldk] (transposed; k >= K zero-filled).
cudaError_t transpose_split_tf32_launch(const double *src, float *hi,
                                        float *lo, int64_t P, int K,
                                        int64_t N, int64_t ldn, int64_t ldk,
                                        cudaStream_t st);

// ---- emulated FP64 preparation (see prep.cu) --------------------------------
cudaError_t rowmax_launch(const double *src, int64_t npq, int64_t R, int64_t K,
                          int64_t kp, unsigned long long *rmax,
                          cudaStream_t st);
cudaError_t colmax_launch(const double *src, int64_t P, int64_t K, int64_t N,
                          int64_t w, int64_t wsrc, int64_t ldsrc,
                          unsigned long long *cmax, cudaStream_t st);
cudaError_t exps_launch(const unsigned long long *m1,
                        const unsigned long long *m2, double s2, int64_t n,
                        signed char *e, cudaStream_t st);
cudaError_t slice_a_launch(const double *src, int64_t npq, int64_t R,
                           int64_t K, int64_t kp, int64_t kpi, double scale,
                           const signed char *ea, int S, signed char *out,
                           cudaStream_t st);
cudaError_t slice_b_launch(const double *src, int64_t P, int K, int64_t N,
                           int64_t w, int64_t wsrc, int64_t ldsrc, int64_t kpi,
                           double scale, const signed char *eb, int S,
                           signed char *out, cudaStream_t st);

}  // namespace ptb
