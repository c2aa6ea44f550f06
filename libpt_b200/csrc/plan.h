// Internal plan object behind the libpt_plan_* C API.
#pragma once

#include <string>
#include <vector>

#include "engine.h"
#include "exec.h"
#include "pt.h"

namespace ptb {

void set_error(const std::string &msg);
const char *last_error();

// Returns a LIBPT_ERR_* status (after recording the message) when a CUDA
// runtime call fails.
#define CK(call)                                                          \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      ::ptb::set_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
      return e_ == cudaErrorMemoryAllocation ? LIBPT_ERR_NOMEM            \
                                             : LIBPT_ERR_CUDA;            \
    }                                                                     \
  } while (0)
// Host allocations through the libpt_set_malloc / libpt_set_free hooks.
void *host_alloc(size_t n);
void host_free(void *p);

// Symbolic occupied index of a job segment: 0 = i, 1 = j, 2 = k.
struct SegT {
  int16_t amap, bmap, neg;
  int8_t aq, ap, bp;
  int32_t ksteps;   // ceil(k / GEMM_BK) for the DMMA kernel
  int32_t k;        // contraction length of the segment
};

// What a map index of a case views: an A operand [P][Q][R][pad4(K)] or a B
// operand [P][K][Nld] (first N columns meaningful) of padded FP64 data.
struct OpDesc {
  int role = -1;    // 0: A, 1: B, -1: unused
  const double *src = nullptr;
  int64_t K = 0, R = 0, Q = 0, P = 0, N = 0, Nld = 0;
  // B source geometry: element (p, k, n) at src[(p K + k) ldsrc + col(n)],
  // col(n) = (n / w) wsrc + n % w, zero when n % w >= wsrc
  int64_t ldsrc = 0, w = 0, wsrc = 0;
  // emulated FP64: scale family (operands of one job side share row / column
  // scales) and part (0: amplitude x OVVV product, 1: OOVO x amplitude)
  int fam = -1, part = 0;
};

// TF32 hi/lo planes of one operand, in tensor-core layout.
struct Planes {
  float *hi = nullptr, *lo = nullptr;
};

// Emulated-FP64 state of one scale family.
struct Family {
  int id = -1;
  int64_t n = 0;                          // rows (A) or columns (B)
  unsigned long long *max0 = nullptr;     // per row/column |max| of part 0
  unsigned long long *max1 = nullptr;     // ... of part 1
  signed char *e = nullptr;               // joint exponents
};

struct JobT {
  int64_t off;      // output offset inside the triple's workspace slice
  int32_t M, N;
  int64_t ldc;
  int nseg;
  SegT seg[MAX_SEG];
  const signed char *ea = nullptr, *eb = nullptr;   // emulated FP64 scales
};

// Padded device copies of one amplitude + integral set (index 0 aaaa,
// 1 abab, 2 bbbb, 3 baba; packed pairs 0 aaaa, 1 bbbb).
struct OperandSet {
  double *tau[4] = {nullptr, nullptr, nullptr, nullptr};
  double *taup[2] = {nullptr, nullptr};
  double *ovvv[4] = {nullptr, nullptr, nullptr, nullptr};
  double *oovo[4] = {nullptr, nullptr, nullptr, nullptr};
  // emulated FP64 from device inputs: the caller's pt.h OVVV blocks are
  // sliced in place (no padded FP64 copy); ovvv[] is then null
  const double *ovvv_src[4] = {nullptr, nullptr, nullptr, nullptr};
  int balance = 0;   // OOVO x amplitude products: A scaled 2^-balance, B 2^+
};

struct SpinCase {
  int type = 0;          // 0: same-spin (aaa), 1: mixed-spin (aab)
  int flip = 0;          // aaa: 0 alpha, 1 beta; aab: 0 (a,a,b), 1 (b,b,a)
  int oa = 0, va = 0, ob = 0, vb = 0;   // sizes as seen by this case
  int64_t first = 0, count = 0;         // range in the triples queue
  MapSet maps;
  std::vector<JobT> jobs;               // per-triple job templates
  EpiArgs epi;                          // fixed epilogue arguments
  EpiArgs *d_epi = nullptr;             // ... in device memory
  int64_t ws_stride = 0;                // doubles of contraction output
  int4 *d_tiles = nullptr;
  int ntiles = 0, ctiles = 0;
  CUtensorMap *d_maps = nullptr;        // the kernel's views, device memory
  double flops_per_triple = 0.0;        // reference GEMM flops
  int bm = GEMM_BM;                     // CTA tile rows of this case's GEMMs
  OpDesc opd[MAX_MAPS];                 // operand behind each DMMA map
  TcMapSet tcmaps;                      // tensor-core views (TF32: map 2i,
                                        // 2i+1; emulated FP64: map i)
  signed char *i8pl[MAX_MAPS] = {};     // digit planes behind INT8 map i
};

}  // namespace ptb

// A host-array OVVV block whose copy is deferred: a restricted FP64
// host-array solve streams these by occupied index (rows_per_index rows of
// w elements each) next to the triples that need them.
struct DeferredBlock {
  double *dst;              // padded device block (dpitch per row)
  const char *src;          // the caller's host array
  int64_t rows_per_index, w, dpitch;
};

struct libpt_plan {
  int kind = 0;
  bool unrestricted = false, ft = false;
  int oa = 0, va = 0, ob = 0, vb = 0;
  int dtype = 0, precision = 0;
  cudaStream_t st = nullptr;
  double factor = 1.0;
  // deferred host OVVV copies (plan_run_streamed), their copy stream, the
  // event that orders the triples after them, and the upload staging
  bool defer_ovvv = false;   // record host OVVV copies instead of making them
  std::vector<DeferredBlock> deferred;
  cudaStream_t st_up = nullptr;
  cudaEvent_t ev_up = nullptr;
  void *up_stage[2] = {nullptr, nullptr};
  size_t up_stage_bytes = 0;
  std::vector<void *> allocs;
  ptb::OperandSet L, R;
  double *d_ov = nullptr, *ov1 = nullptr, *ov2 = nullptr;
  bool has_f = true;                    // f_ov / f2_ov not all zero
  double *oovv[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<ptb::SpinCase> cases;
  std::vector<int4> queue;              // (case, i, j, k)
  double *e_slot = nullptr;
  // phase times of creation (s), recorded for LIBPT_PROFILE=1
  double prof_upload = 0, prof_prepare = 0, prof_tune = 0;
  // round resources: contraction outputs (packed by each triple's own
  // size), partial energies and descriptors of one round of triples
  double *ws = nullptr;
  double *partials = nullptr;
  char *d_desc = nullptr;
  int64_t ws_cap = 0, part_cap = 0;     // doubles held
  size_t tri_cap = 0;                   // triples a round may hold
  size_t ws_budget = 0;                 // workspace size limit (bytes)
  int64_t ws_stride = 0;                // max over cases (doubles)
  int64_t ws_stride_min = 0;            // min over cases (doubles)
  int ntiles_max = 0;                   // max epilogue tiles of a triple
  size_t jobs_max = 0;                  // max GEMM jobs of a triple
  unsigned *d_err = nullptr;
  size_t max_batch = 0;                 // 0: derive from the memory budget
  ptb::Executor exec;                   // the plan's own rounds
  bool exec_ready = false;
  // caller-provided device arena: when set, every device buffer of the plan
  // is carved from it and nothing is allocated or freed
  char *arena = nullptr;
  size_t arena_size = 0, arena_used = 0;
  // tensor-core planes, keyed by (source block, role)
  std::vector<std::pair<std::pair<const double *, int>, ptb::Planes>> planes;
  // emulated FP64: digit planes per (source block, role), scale families
  int slices = 6;                       // digit planes the kernels use
  int slices_store = 6;                 // digit planes stored (>= slices)
  int dbits = 7;                        // digit base bits of the planes (7, 8)
  bool slices_auto = false;             // choose slices for emu_tol
  double emu_tol = 1e-6;                // |dE| target of the choice (Eh)
  ptb::I8Tile i8tile{64, ptb::I8_KCHUNK, 0, 0};   // emulated FP64 tile variant
  std::vector<std::pair<std::pair<const double *, int>, signed char *>> i8planes;
  std::vector<ptb::Family> fams;
  // kernel timing (libpt_plan_timing): events around each round's GEMMs
  // and epilogues
  bool timing = false;
  ptb::ExecTiming tm;
  int64_t launches = 0;                      // kernels launched by runs
};

namespace ptb {

// args: pt.h tensors of `kind` in the reference's order; `host` selects host
// (true) or device (false) pointers; dtype 0 = FP64, 1 = FP32.
// arena: carve every device buffer from [arena, arena + arena_size) (no
// allocation); arena_nb caps the triples of one round (0: what fits).
int plan_create(int kind, size_t oa, size_t va, size_t ob, size_t vb,
                const void *const *args, int dtype, int precision, bool host,
                cudaStream_t st, libpt_plan **out, void *arena = nullptr,
                size_t arena_size = 0, size_t arena_nb = 0,
                bool stream_ovvv = false);
// Exact device bytes plan_create takes from an arena for these arguments
// with rounds of up to nb triples (a sizing pass: host logic only, no
// device work); 0 if the arguments are invalid.
size_t plan_footprint(int kind, size_t oa, size_t va, size_t ob, size_t vb,
                      int dtype, int precision, bool host, size_t nb);
// Tensor-core views of TF32 planes (see engine.h): A planes [P][Q][R][Kp],
// B planes [P][N][Kp] (Kp = pad4(K) floats per row).
int tc_map_a(CUtensorMap *m, const float *p, int64_t K, int64_t R, int64_t Q,
             int64_t P);
int tc_map_b(CUtensorMap *m, const float *p, int64_t K, int64_t N, int64_t P);
// INT8 digit-plane views: A planes [2S][P][Q][kpi/32][R][32] as
// (32, R, kpi/32, Q*P, 2S), B planes [S][P][kpi/32][N][32] as
// (32, N, kpi/32, P, S); kpi = i8_kpad(K).  Boxes of 32 bytes x 128 (A) or
// bn (B) rows, swizzled to 32 bytes.
int i8_map_a(CUtensorMap *m, const signed char *p, int64_t K, int64_t R,
             int64_t Q, int64_t P, int S);
int i8_map_b(CUtensorMap *m, const signed char *p, int64_t K, int64_t N,
             int64_t P, int S, int bn);
// DMMA views of padded FP64 blocks: A [P][Q][R][pad4(K)], B [P][K][Nld].
int dmma_map_a(CUtensorMap *m, const double *p, int64_t K, int64_t R,
               int64_t Q, int64_t P, int bm);
int dmma_map_b(CUtensorMap *m, const double *p, int64_t N, int64_t Nld,
               int64_t K, int64_t P);
int plan_run(libpt_plan *p, const int64_t *idx, size_t n);
// The whole queue; with deferred OVVV copies, each occupied index's rows are
// copied on a second stream while the triples whose indices are all below it
// run (same energies: each triple writes its own slot).
int plan_run_streamed(libpt_plan *p);
// Where the next triple of a plan goes in its round resources, and the end
// of the region this round may use (negative / zero: the plan's capacity),
// so two rounds of one plan can be in flight in disjoint halves.
struct PlanCursor {
  int64_t ws = 0, part = 0;
  size_t triples = 0;
  int64_t ws_end = -1, part_end = -1;
  size_t tri_end = 0;
};
// Appends queue entries ents[0..n) of plan p to a round while they fit the
// plan's round resources (from cur on); *taken = entries appended.
int plan_append(libpt_plan *p, const int64_t *ents, size_t n, PlanCursor &cur,
                Round &r, size_t *taken);
// The GEMM variant that runs a plan's spin case.
GemmGroup plan_group(const libpt_plan *p, const SpinCase &c);
// Reads the per-triple energies back on stream rs (null: the plan's) and
// sums them in queue order (restricted factor applied).
int plan_energy(libpt_plan *p, const int64_t *idx, size_t n, double *e,
                cudaStream_t rs = nullptr);
// Queue-order compensated sum of slots[idx[0..n)] (idx NULL: all `total`),
// without the restricted factor; the sum libpt_plan_energy applies.
int sum_slots(const double *slots, size_t total, const int64_t *idx, size_t n,
              double *out);
// Monotonic wall clock (s); LIBPT_PROFILE=1 in the environment.
double wall_seconds();
bool profile_enabled();
// Entries of queue length `total` that rank `rank` of `size` owns (q % size
// == rank); writes them to idx when non-NULL; -1 for invalid arguments.
int64_t shard_entries(int64_t total, int rank, int size, int64_t *idx);
// Zeroes every energy slot, then runs the entries rank `rank` owns.
int plan_run_shard(libpt_plan *p, int rank, int size);
void plan_destroy(libpt_plan *p);
double plan_flops(const libpt_plan *p, int64_t first, int64_t n);
int plan_kernel_stats(libpt_plan *p, double *gemm_ms, int64_t *gemm_launches,
                      double *gemm_flops, double *epi_ms, int64_t *launches);

}  // namespace ptb
