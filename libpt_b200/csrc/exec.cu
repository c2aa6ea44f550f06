// Round executor (see exec.h).
#include "exec.h"

#include <algorithm>
#include <cstring>
#include <tuple>

#include "plan.h"
#include "pt.h"

namespace ptb {

bool GemmGroup::operator<(const GemmGroup &o) const {
  return std::tie(kind, bm, slices, tile.bn, tile.kc, tile.pair, tile.ts) <
         std::tie(o.kind, o.bm, o.slices, o.tile.bn, o.tile.kc, o.tile.pair,
                  o.tile.ts);
}

std::string GemmGroup::name() const {
  return std::to_string(kind) + "/" + std::to_string(bm) + "/" +
         std::to_string(slices) + "/" + std::to_string(tile.bn) + "/" +
         std::to_string(tile.kc) + (tile.pair ? "/pair" : "") +
         (tile.ts ? "/ts" : "");
}

int GroupMaps::add(const CUtensorMap *d, const CUtensorMap *h, int n) {
  for (size_t x = 0; x < dev.size(); ++x)
    if (dev[x] == d) return first[x];
  dev.push_back(d);
  host.push_back(h);
  count.push_back(n);
  first.push_back(total);
  total += n;
  return first.back();
}

void Round::clear() {
  gemm.clear();
  maps.clear();
  for (int a = 0; a < 2; ++a)
    for (int f = 0; f < 2; ++f) {
      epi[a][f].clear();
      epi_blocks[a][f].clear();
      epi_hasf[a][f] = false;
    }
  red.clear();
  gemm_flops = 0.0;
  triples = 0;
}

void ExecTiming::clear() {
  for (cudaEvent_t e : ev_gemm) cudaEventDestroy(e);
  for (cudaEvent_t e : ev_epi) cudaEventDestroy(e);
  ev_gemm.clear();
  ev_epi.clear();
  flops.clear();
}

namespace {

// Fixed header slots at the start of the descriptor buffer.
constexpr size_t SLOT = 32;
constexpr size_t HDR = 512;
static_assert(sizeof(GemmList) <= SLOT && sizeof(EpiList) <= SLOT &&
                  sizeof(RedList) <= SLOT,
              "list headers fit their slots");
static_assert((EXEC_MAX_GROUPS + 4 + 1) * SLOT <= HDR, "header size");

size_t gemm_slot(int g) { return g * SLOT; }
size_t epi_slot(int aab, int ft) {
  return (EXEC_MAX_GROUPS + 2 * aab + ft) * SLOT;
}
size_t red_slot() { return (EXEC_MAX_GROUPS + 4) * SLOT; }
size_t align64(size_t x) { return (x + 63) & ~size_t(63); }

constexpr int RED_GRID = 148 * 8;

}  // namespace

int Executor::init(cudaStream_t st, void *d_buf, size_t cap, bool graphs,
                   size_t triples, size_t jobs_per_triple) {
  st_ = st;
  d_buf_ = static_cast<char *>(d_buf);
  cap_ = cap;
  graphs_ = graphs;
  slot_jobs_ = triples * jobs_per_triple;
  if (graphs_ && bytes_for(triples, jobs_per_triple, true) > cap_) {
    set_error("executor: descriptor buffer smaller than its fixed layout");
    return LIBPT_ERR_ARG;
  }
  for (int a = 0; a < 2; ++a)
    for (int f = 0; f < 2; ++f) epi_grid_[a][f] = 148 * epi_blocks_per_sm(a, f);
  if (graphs_) {
    for (int b = 0; b < 2; ++b) {
      if (cudaHostAlloc((void **)&h_buf_[b], cap_, cudaHostAllocDefault) !=
          cudaSuccess) {
        set_error("executor: pinned staging allocation failed");
        return LIBPT_ERR_NOMEM;
      }
      if (cudaEventCreateWithFlags(&copied_[b], cudaEventDisableTiming) !=
          cudaSuccess)
        return LIBPT_ERR_CUDA;
    }
  }
  return LIBPT_OK;
}

void Executor::destroy() {
  for (auto &kv : cache_) cudaGraphExecDestroy(kv.second);
  cache_.clear();
  for (int b = 0; b < 2; ++b) {
    if (h_buf_[b]) cudaFreeHost(h_buf_[b]);
    if (copied_[b]) cudaEventDestroy(copied_[b]);
    h_buf_[b] = nullptr;
    copied_[b] = nullptr;
  }
}

size_t Executor::bytes_for(size_t triples, size_t jobs_per_triple,
                           bool graphs) {
  const size_t jobs = triples * jobs_per_triple * sizeof(GemmJob);
  return HDR + 64 * (EXEC_MAX_GROUPS + 5) +
         (graphs ? EXEC_MAX_GROUPS : 1) * jobs +
         triples * (sizeof(EpiItem) + sizeof(RedItem));
}

int Executor::launch_all(const std::vector<GemmGroup> &groups,
                         unsigned *d_err, const bool epi_on[2][2],
                         ExecTiming *timing, const Round *r,
                         int64_t *launches) {
  // grids: fixed for graph replay, trimmed to the work for direct launches
  const bool fixed = r == nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (timing)
    for (int x = 0; x < 4; ++x) CK(cudaEventCreate(&ev[x]));
  if (timing) CK(cudaEventRecord(ev[0], st_));
  int g = 0;
  for (const GemmGroup &grp : groups) {
    GemmList *lst = reinterpret_cast<GemmList *>(d_buf_ + gemm_slot(g));
    int grid = GEMM_GRID;
    if (!fixed) {
      int tiles = 0;
      for (const GemmJob &j : r->gemm.at(grp)) tiles += j.mtiles * j.ntiles_n;
      grid = std::min(GEMM_GRID, tiles);
    }
    // direct launches whose views fit take them as kernel parameters
    const LaunchMaps *pm = nullptr;
    if (!fixed) {
      const GroupMaps &gm = r->maps.at(grp);
      if (gm.total <= LAUNCH_MAPS) {
        for (size_t x = 0; x < gm.host.size(); ++x)
          std::memcpy(&pmaps_.m[gm.first[x]], gm.host[x],
                      gm.count[x] * sizeof(CUtensorMap));
        pm = &pmaps_;
      }
    }
    const GemmJob *jobs = gjobs_[g];
    int njobs = 0, ntiles = 0;
    if (!fixed) {
      const std::vector<GemmJob> &v = r->gemm.at(grp);
      njobs = (int)v.size();
      for (const GemmJob &j : v) ntiles += j.mtiles * j.ntiles_n;
    }
    if (grid > 0) {
      if (grp.kind == 0) {
        CK(gemm_dmma_launch(jobs, lst, njobs, ntiles, pm, grp.bm, grid, d_err,
                            st_));
      } else if (grp.kind == 1) {
        TcProducts pr;
        memset(&pr, 0, sizeof(pr));
        const int8_t pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};   // hh + hl + lh
        for (int q = 0; q < 3; ++q) {
          pr.pa[q] = pa[q];
          pr.pb[q] = pb[q];
          pr.acc[q] = 0;
        }
        pr.n = 3;
        CK(gemm_tc_launch(jobs, lst, njobs, ntiles, pm, grid, pr, d_err, st_));
      } else {
        CK(gemm_i8_launch(grp.slices, grp.tile, jobs, lst, njobs, ntiles, pm,
                          grid, d_err, st_));
      }
      if (launches) ++*launches;
    }
    ++g;
  }
  if (timing) {
    CK(cudaEventRecord(ev[1], st_));
    CK(cudaEventRecord(ev[2], st_));
  }
  for (int a = 0; a < 2; ++a)
    for (int f = 0; f < 2; ++f) {
      if (!epi_on[a][f]) continue;
      const EpiList *lst = reinterpret_cast<const EpiList *>(d_buf_ + epi_slot(a, f));
      int grid = epi_grid_[a][f], nitems = 1;
      if (!fixed) {   // one CTA per (tile, item)
        grid = 0;
        for (int b : r->epi_blocks[a][f]) grid = std::max(grid, b);
        nitems = (int)r->epi[a][f].size();
      }
      if (grid <= 0) continue;
      const bool hasf = fixed || r->epi_hasf[a][f];
      const EpiItem *items = fixed ? nullptr : epi_items_[a][f];
      CK(a ? epi_aab_launch(lst, items, f, hasf, grid, nitems, fixed, st_)
           : epi_aaa_launch(lst, items, f, hasf, grid, nitems, fixed, st_));
      if (launches) ++*launches;
    }
  {
    const RedList *lst = reinterpret_cast<const RedList *>(d_buf_ + red_slot());
    int grid = fixed ? RED_GRID : std::min<int>(RED_GRID, (int)r->red.size());
    if (grid > 0) {
      CK(reduce_partials_launch(lst, grid, st_));
      if (launches) ++*launches;
    }
  }
  if (timing) {
    CK(cudaEventRecord(ev[3], st_));
    timing->ev_gemm.push_back(ev[0]);
    timing->ev_gemm.push_back(ev[1]);
    timing->ev_epi.push_back(ev[2]);
    timing->ev_epi.push_back(ev[3]);
    timing->flops.push_back(r ? r->gemm_flops : 0.0);
  }
  return LIBPT_OK;
}

int Executor::run(Round &r, unsigned *d_err, ExecTiming *timing,
                  int64_t *launches, bool replay) {
  if (r.empty()) return LIBPT_OK;
  std::vector<GemmGroup> groups;
  for (auto &kv : r.gemm)
    if (!kv.second.empty()) groups.push_back(kv.first);
  if ((int)groups.size() > EXEC_MAX_GROUPS) {
    set_error("executor: too many GEMM variants in one round");
    return LIBPT_ERR_ARG;
  }
  // layout and flat numbering (graphs: job arrays in fixed slots)
  size_t off = HDR;
  std::vector<size_t> goff(groups.size());
  const size_t slot_bytes = align64(slot_jobs_ * sizeof(GemmJob));
  gjobs_.resize(groups.size());
  for (size_t g = 0; g < groups.size(); ++g) {
    std::vector<GemmJob> &jobs = r.gemm[groups[g]];
    int tiles = 0;
    for (GemmJob &j : jobs) {
      j.tile_begin = tiles;
      tiles += j.mtiles * j.ntiles_n;
    }
    if (graphs_ && jobs.size() > slot_jobs_) {
      set_error("executor: GEMM jobs exceed their graph slot");
      return LIBPT_ERR_ARG;
    }
    goff[g] = graphs_ ? HDR + g * slot_bytes : off;
    gjobs_[g] = reinterpret_cast<const GemmJob *>(d_buf_ + goff[g]);
    off = graphs_ ? HDR + EXEC_MAX_GROUPS * slot_bytes
                  : align64(off + jobs.size() * sizeof(GemmJob));
  }
  if (graphs_) off = std::max(off, HDR + EXEC_MAX_GROUPS * slot_bytes);
  size_t eoff[2][2];
  bool epi_on[2][2];
  for (int a = 0; a < 2; ++a)
    for (int f = 0; f < 2; ++f) {
      int blocks = 0;
      for (size_t x = 0; x < r.epi[a][f].size(); ++x) {
        r.epi[a][f][x].block_begin = blocks;
        r.epi[a][f][x].nblk = r.epi_blocks[a][f][x];
        blocks += r.epi_blocks[a][f][x];
      }
      epi_on[a][f] = blocks > 0;
      eoff[a][f] = off;
      off = align64(off + r.epi[a][f].size() * sizeof(EpiItem));
    }
  const size_t roff = off;
  off = align64(off + r.red.size() * sizeof(RedItem));
  if (off > cap_) {
    set_error("executor: round descriptors exceed the buffer (" +
              std::to_string(off) + " > " + std::to_string(cap_) + " bytes)");
    return LIBPT_ERR_NOMEM;
  }
  // host image
  char *h;
  if (graphs_) {
    CK(cudaEventSynchronize(copied_[parity_]));   // its previous copy is done
    h = h_buf_[parity_];
  } else {
    if (staging_.size() < off) staging_.resize(off);
    h = staging_.data();
  }
  memset(h, 0, HDR);
  for (size_t g = 0; g < groups.size(); ++g) {
    const std::vector<GemmJob> &jobs = r.gemm[groups[g]];
    std::memcpy(h + goff[g], jobs.data(), jobs.size() * sizeof(GemmJob));
    GemmList l{};
    l.jobs = reinterpret_cast<const GemmJob *>(d_buf_ + goff[g]);
    l.njobs = (int32_t)jobs.size();
    l.ntiles = jobs.empty() ? 0
                            : jobs.back().tile_begin +
                                  jobs.back().mtiles * jobs.back().ntiles_n;
    std::memcpy(h + gemm_slot((int)g), &l, sizeof(l));
  }
  for (int a = 0; a < 2; ++a)
    for (int f = 0; f < 2; ++f) {
      const std::vector<EpiItem> &it = r.epi[a][f];
      std::memcpy(h + eoff[a][f], it.data(), it.size() * sizeof(EpiItem));
      EpiList l;
      l.items = reinterpret_cast<const EpiItem *>(d_buf_ + eoff[a][f]);
      epi_items_[a][f] = l.items;   // direct launches take it as a parameter
      l.nitems = (int32_t)it.size();
      l.nblocks = it.empty() ? 0
                             : it.back().block_begin + r.epi_blocks[a][f].back();
      std::memcpy(h + epi_slot(a, f), &l, sizeof(l));
    }
  {
    std::memcpy(h + roff, r.red.data(), r.red.size() * sizeof(RedItem));
    RedList l;
    l.items = reinterpret_cast<const RedItem *>(d_buf_ + roff);
    l.nitems = (int32_t)r.red.size();
    l.pad_ = 0;
    std::memcpy(h + red_slot(), &l, sizeof(l));
  }
  CK(cudaMemcpyAsync(d_buf_, h, off, cudaMemcpyHostToDevice, st_));
  if (graphs_) {
    CK(cudaEventRecord(copied_[parity_], st_));
    parity_ ^= 1;
  }
  if (!graphs_ || timing || !replay)
    return launch_all(groups, d_err, epi_on, timing, &r, launches);
  // graph replay keyed by the variant set
  std::string key;
  for (const GemmGroup &g : groups) key += g.name() + ";";
  for (int a = 0; a < 2; ++a)
    for (int f = 0; f < 2; ++f) key += epi_on[a][f] ? "1" : "0";
  auto it = cache_.find(key);
  if (it == cache_.end()) {
    // first round of this variant set: launch directly, then capture the
    // same sequence (fixed grids) for the rounds that follow
    if (int e = launch_all(groups, d_err, epi_on, nullptr, &r, launches))
      return e;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
    const int e = launch_all(groups, d_err, epi_on, nullptr, nullptr, nullptr);
    cudaError_t ce = cudaStreamEndCapture(st_, &graph);
    if (e) return e;
    if (ce != cudaSuccess) {
      set_error(std::string("graph capture: ") + cudaGetErrorString(ce));
      return LIBPT_ERR_CUDA;
    }
    cudaGraphExec_t exec;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
      set_error(std::string("graph instantiate: ") + cudaGetErrorString(ce));
      return LIBPT_ERR_CUDA;
    }
    cache_[key] = exec;
    return LIBPT_OK;
  }
  CK(cudaGraphLaunch(it->second, st_));
  ++replays_;
  if (launches) {
    *launches += (int64_t)groups.size() + 1;
    for (int a = 0; a < 2; ++a)
      for (int f = 0; f < 2; ++f) *launches += epi_on[a][f];
  }
  return LIBPT_OK;
}

}  // namespace ptb
