// Round executor: one "round" is a set of triples, possibly from many plans,
// run as one launch per kernel variant (GEMM groups, then the energy
// epilogues, then the per-triple reductions).  All work lists live in one
// device descriptor buffer written by a single host-to-device copy; every
// kernel reads its list from fixed slots there, so the launch sequence of a
// given variant set can be captured once as a CUDA graph and replayed for
// every later round with the same variants.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "engine.h"

namespace ptb {

// One GEMM launch variant.
struct GemmGroup {
  int kind = 0;        // 0: FP64 DMMA, 1: 3xTF32, 2: emulated FP64 (INT8)
  int bm = 128;        // DMMA tile rows
  int slices = 0;      // INT8 digit planes
  I8Tile tile{0, 0};   // INT8 tile shape
  bool operator<(const GemmGroup &o) const;
  std::string name() const;
};

constexpr int EXEC_MAX_GROUPS = 8;   // GEMM variants in one round

// The tensor-map tables a GEMM launch's jobs use (one per plan spin case):
// device copies (for device-memory maps) and host copies (gathered into the
// kernel-parameter table when they fit).
struct GroupMaps {
  std::vector<const CUtensorMap *> dev, host;
  std::vector<int> count, first;
  int total = 0;
  // offset of this case's table in the launch's parameter table
  int add(const CUtensorMap *d, const CUtensorMap *h, int n);
};

struct Round {
  std::map<GemmGroup, std::vector<GemmJob>> gemm;   // tile_begin unset
  std::map<GemmGroup, GroupMaps> maps;
  std::vector<EpiItem> epi[2][2];                   // [aab][ft], block_begin unset
  std::vector<int> epi_blocks[2][2];                // blocks of each item
  bool epi_hasf[2][2] = {};                         // some item's f_ov != 0
  std::vector<RedItem> red;
  double gemm_flops = 0.0;                          // reference flops
  size_t triples = 0;
  void clear();
  bool empty() const { return triples == 0; }
};

// Kernel time of the rounds run while timing is on.
struct ExecTiming {
  std::vector<cudaEvent_t> ev_gemm, ev_epi;   // start / stop pairs
  std::vector<double> flops;
  void clear();
};

class Executor {
 public:
  // d_buf / cap: device memory for the descriptors (owned by the caller);
  // graphs: replay captured CUDA graphs (needs pinned staging, allocated
  // here with cudaHostAlloc) instead of direct launches; the GEMM job
  // arrays then sit at fixed offsets, sized for rounds of up to `triples`
  // triples of up to `jobs_per_triple` jobs (kernels take them as
  // parameters, which a graph fixes).
  int init(cudaStream_t st, void *d_buf, size_t cap, bool graphs,
           size_t triples = 0, size_t jobs_per_triple = 0);
  void destroy();
  // Bytes of descriptors a round of `triples` triples with up to
  // `jobs_per_triple` GEMM jobs each needs (graphs: the fixed layout).
  static size_t bytes_for(size_t triples, size_t jobs_per_triple,
                          bool graphs = false);
  // Launches the round on the stream (asynchronous).  d_err: device error
  // word the kernels set on a timed-out wait.  Returns the kernels launched.
  // replay: use (or capture) the CUDA graph of the round's variant set
  // (graph-capable executors only); otherwise launch directly.
  int run(Round &r, unsigned *d_err, ExecTiming *timing, int64_t *launches,
          bool replay = true);
  int64_t graph_replays() const { return replays_; }
  cudaStream_t stream() const { return st_; }

 private:
  int launch_all(const std::vector<GemmGroup> &groups, unsigned *d_err,
                 const bool epi_on[2][2], ExecTiming *timing,
                 const Round *r, int64_t *launches);
  cudaStream_t st_ = nullptr;
  char *d_buf_ = nullptr;
  size_t cap_ = 0;
  bool graphs_ = false;
  char *h_buf_[2] = {nullptr, nullptr};
  cudaEvent_t copied_[2] = {nullptr, nullptr};
  int parity_ = 0;
  std::vector<char> staging_;
  std::map<std::string, cudaGraphExec_t> cache_;
  LaunchMaps pmaps_;   // staging of a launch's parameter-table maps
  size_t slot_jobs_ = 0;                 // graphs: jobs per GEMM slot
  int64_t replays_ = 0;
  std::vector<const GemmJob *> gjobs_;   // device job arrays of the groups
  int epi_grid_[2][2] = {{0, 0}, {0, 0}};
  const EpiItem *epi_items_[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
};

}  // namespace ptb
