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
  int16_t neg;          // neg != 0: subtract this product (INT8: the index
                        // of the first negated digit plane)
  int16_t half_last;    // INT8: the last K chunk holds <= 32 bytes of K, so
                        // its second MMA K step (all zero) is skipped
  int32_t a_q, a_p;     // A-view coordinates of dims 2 and 3
  int32_t b_p;          // B-view coordinate of dim 2
  int32_t ksteps;       // ceil(K_s / GEMM_BK)
};

struct GemmJob {
  double *out;          // C, row-major with leading dimension ldc
  int64_t ldc;
  int32_t M, N;         // N <= ldc, N % 4 == 0
  int32_t ntiles_n;     // ceil(N / tile columns)
  int32_t tile_begin;   // first flat tile index of this job in the launch
  int32_t nseg;
  int32_t mtiles;       // ceil(M / BM); tiles are numbered M-tile fastest
  GemmSeg seg[MAX_SEG];
  // emulated FP64: power-of-two exponents of the output rows / columns
  const signed char *ea, *eb;
  // The tensor maps (TMA views) the segments' amap / bmap index, in one of
  // two places, chosen per launch: a kernel-parameter table (LaunchMaps,
  // this job's views from entry map0 on; fastest descriptor access), or
  // 64-byte aligned CUtensorMaps in device memory at `maps` (any number of
  // plans per launch, fixed kernel parameters for graph replay; kernels
  // fence each such map before first use).
  const CUtensorMap *maps;
  int32_t map0;
  // emulated FP64: digit base bits of the planes (7 or 8; 0 reads as 7)
  int32_t dbits;
};

// Kernel-parameter table of the tensor maps of one launch (12 KiB of
// parameters: CUDA 12.1+ kernels take up to 32 KiB).
constexpr int LAUNCH_MAPS = 96;
struct LaunchMaps {
  CUtensorMap m[LAUNCH_MAPS];
};

// Work list of one GEMM launch, read by the kernel from device memory so a
// launch's parameters (and a captured CUDA graph) stay fixed while the list
// changes.  Jobs are sorted by tile_begin; ntiles = total tiles.  Kernels
// also take the jobs array itself as a (restrict) parameter, equal to
// list->jobs, so the compiler may keep job fields across their stores.
// The list is also the launch's tile queue: the CTAs of the DMMA and the
// one-CTA INT8 kernels take tiles by incrementing `next` (the reference's
// schedule(dynamic) over triples, src/pt.c:228, 353, on the device), and the
// last CTA to finish resets `next` and `done` to zero for the next launch of
// the same list; the host writes both as zero.
struct GemmList {
  const GemmJob *jobs;
  int32_t njobs, ntiles;
  int32_t next, done;
};

// Persistent grid of the GEMM kernels (one CTA per SM).
constexpr int GEMM_GRID = 148;

size_t gemm_smem_bytes(int bm);
// bm: CTA tile rows, 96 or 128 (the A views' box height must match).  The
// kernels run `grid` persistent CTAs over the list's tiles.  Two forms:
//   pm != null: the launch's tensor maps and the job / tile counts (njobs,
//               ntiles) as kernel parameters (direct launches);
//   pm == null: maps in device memory (GemmJob::maps) and the counts read
//               from d_list (fixed parameters: CUDA graph replay).
cudaError_t gemm_dmma_launch(const GemmJob *d_jobs, GemmList *d_list,
                             int njobs, int ntiles, const LaunchMaps *pm,
                             int bm, int grid, unsigned *d_err,
                             cudaStream_t st);

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

struct MapSet {
  CUtensorMap m[MAX_MAPS];
};

struct TcMapSet {
  CUtensorMap m[TC_MAX_MAPS];
};

struct TcProducts {           // acc[c] += A_plane[pa] * B_plane[pb]^T
  int8_t pa[16], pb[16], acc[16];
  int n;
};

int tc_kchunk_elems(int kind);   // K elements per pipeline stage (TF32)
// 3xTF32: planes {hi, lo} in separate maps (2i, 2i+1), products from prods.
cudaError_t gemm_tc_launch(const GemmJob *d_jobs, GemmList *d_list,
                           int njobs, int ntiles, const LaunchMaps *pm,
                           int grid, const TcProducts &prods, unsigned *d_err,
                           cudaStream_t st);

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
  int bn;     // tile columns (multiple of 16, S * bn <= 512)
  int kc;     // K bytes per pipeline stage (I8_KCHUNK: two MMA K steps)
  int pair;   // 1: a CTA pair (two SMs) computes a 256 x bn tile, each CTA
              // loading its 128 rows of A and half of the bn columns of B
  int ts;     // 1: the MMAs read A from TMEM (copied there once per plane
              // and K step) instead of re-reading it from shared memory
};
// Digit planes are stored in K chunks of I8_KCHUNK bytes (64: one 64-byte
// swizzled row per TMA box row; a box of R rows is one contiguous block).
constexpr int I8_KCHUNK = 64;
// K padded to whole chunks: the row extent of the digit planes.
inline int64_t i8_kpad(int64_t K) {
  return (K + I8_KCHUNK - 1) & ~int64_t(I8_KCHUNK - 1);
}
// The tile variants compiled for a slice count (widest first); returns
// their number (0 for an unsupported count).
int i8_tiles(int slices, const I8Tile **out);
cudaError_t gemm_i8_launch(int slices, I8Tile tile, const GemmJob *d_jobs,
                           GemmList *d_list, int njobs, int ntiles,
                           const LaunchMaps *pm, int grid, unsigned *d_err,
                           cudaStream_t st);

// ---- energy epilogues ------------------------------------------------------

constexpr int EPI_A = 8, EPI_B = 8, EPI_C = 32;   // tile extents a x b x c
constexpr int EPI_THREADS = 256;
constexpr int EPI_CS = EPI_C + 2;                 // smem row stride (banks)

// Fixed arguments of one spin case's epilogue (device memory, per plan).
struct EpiArgs {
  int64_t offL[3];        // array offsets of the (first) amplitude W / L
  int64_t offR[3];        // offsets of R for (fT); offR[0] < 0 for (T)
  int64_t ld[3];          // leading dims: aaa {ldT}; aab {ldU1, ldU2, ldP}
  int64_t rowU1, rowU2;   // aab: padded inner extents of U1 (vb) and U2 (va)
  int oa, va, ob, vb;
  const double *d_a, *d_b;                  // denominators [o][v]
  const double *ov1_a, *ov1_b;              // t1 / l1
  const double *g1_ab, *g1_aa;              // i_oovv blocks
  int64_t g1_ld_ab, g1_ld_aa;               // their inner leading dims
  const double *ov2_a, *ov2_b;              // f_ov / f2_ov
  const double *g2_ab, *g2_aa;              // t2 / l2 blocks
  int64_t g2_ld_ab, g2_ld_aa;
  int ntiles;             // CTA tiles of one triple
  const int4 *tiles;      // aaa: (a0, b0, c0); aab: (a0, b0, 0) block pairs
  int ctiles;             // aab: number of c blocks
  int has_f;              // f_ov / f2_ov has a nonzero entry (else its
                          // disconnected-term products are skipped)
};

// One triple of an epilogue launch.
struct EpiItem {
  const EpiArgs *args;    // its spin case's arguments
  const double *ws;       // its contraction outputs
  double *partials;       // its per-tile partial energies [args->ntiles]
  int32_t i, j, k;
  int32_t block_begin;    // first flat CTA tile of this item in the launch
  int32_t nblk;           // its CTA tiles (args->ntiles)
  int32_t pad_;
};

struct EpiList {          // items sorted by block_begin
  const EpiItem *items;
  int32_t nitems, nblocks;
};

// One triple's fixed-order reduction: *dst = sum of partials[0..n).
struct RedItem {
  const double *partials;
  double *dst;
  int32_t n, pad_;
};

struct RedList {
  const RedItem *items;
  int32_t nitems, pad_;
};

size_t epi_smem_bytes(bool aab, bool ft);
// persistent: `grid` CTAs stride over list->nblocks tiles (a fixed grid,
// for graph replay); otherwise a (max tiles of an item) x (items) grid, one
// CTA per tile, grid = max tiles and nitems the item count, whose CTAs read
// their item from d_items (the list's item array, passed directly so that
// the tile's first load does not wait for the list).
cudaError_t epi_aaa_launch(const EpiList *d_list, const EpiItem *d_items,
                           bool ft, bool hasf, int grid, int nitems,
                           bool persistent, cudaStream_t st);
cudaError_t epi_aab_launch(const EpiList *d_list, const EpiItem *d_items,
                           bool ft, bool hasf, int grid, int nitems,
                           bool persistent, cudaStream_t st);
// CTAs the epilogue keeps resident per SM (for persistent grids).
int epi_blocks_per_sm(bool aab, bool ft);
cudaError_t reduce_partials_launch(const RedList *d_list, int grid,
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
// Digit planes of base 2^bits (7: balanced digits; 8: signed top digit,
// unsigned lower digits, the last rounded); see prep.cu.
cudaError_t slice_a_launch(const double *src, int64_t npq, int64_t R,
                           int64_t K, int64_t kp, int64_t kpi, double scale,
                           const signed char *ea, int S, int bits,
                           signed char *out, cudaStream_t st);
cudaError_t slice_b_launch(const double *src, int64_t P, int K, int64_t N,
                           int64_t w, int64_t wsrc, int64_t ldsrc, int64_t kpi,
                           double scale, const signed char *eb, int S, int bits,
                           signed char *out, cudaStream_t st);

}  // namespace ptb
