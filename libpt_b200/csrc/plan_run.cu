// Running a plan's triples: round resources, appending queue entries to a
// round, the rounds of a run, the energy read-back and its fixed-order
// compensated sum, and the sharded run over ranks (src/pt.c:213,
// 474-477).
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
#include <ctime>

namespace ptb {

// Sizes the round resources for `ents` (up to the workspace budget): the
// contraction outputs of every triple, their partial energies and the
// round descriptors.
int ensure_capacity(libpt_plan *p, const std::vector<int64_t> &ents) {
  int64_t want = 0, biggest = 0;
  for (int64_t q : ents) {
    const int64_t st = p->cases[p->queue[q].x].ws_stride;
    want += st;
    biggest = std::max(biggest, st);
    if (want * 8 >= (int64_t)p->ws_budget) break;
  }
  if (p->arena) {   // fixed resources: rounds are cut to what they hold
    if (p->tri_cap >= 1 && biggest <= p->ws_cap) return LIBPT_OK;
    set_error("scratch arena workspace smaller than one triple");
    return LIBPT_ERR_NOMEM;
  }
  want = std::max(std::min<int64_t>(want, (int64_t)(p->ws_budget / 8)), biggest);
  const size_t tri = std::max<size_t>(
      1, std::min<size_t>({(size_t)4096, ents.size(),
                           (size_t)(want / std::max<int64_t>(p->ws_stride_min, 1))}));
  if (want <= p->ws_cap && tri <= p->tri_cap) return LIBPT_OK;
  CK(cudaStreamSynchronize(p->st));
  for (void **q : {(void **)&p->ws, (void **)&p->partials, (void **)&p->d_desc}) {
    if (!*q) continue;
    auto it = std::find(p->allocs.begin(), p->allocs.end(), *q);
    if (it != p->allocs.end()) p->allocs.erase(it);
    cudaFree(*q);
    *q = nullptr;
  }
  if (p->exec_ready) {
    p->exec.destroy();
    p->exec_ready = false;
  }
  p->ws_cap = p->part_cap = 0;
  p->tri_cap = 0;
  const int64_t part = (int64_t)tri * std::max(p->ntiles_max, 1);
  const size_t desc = Executor::bytes_for(tri, p->jobs_max);
  if (dalloc(p, (void **)&p->ws, want * 8) ||
      dalloc(p, (void **)&p->partials, part * 8) ||
      dalloc(p, (void **)&p->d_desc, desc))
    return LIBPT_ERR_NOMEM;
  if (int r = p->exec.init(p->st, p->d_desc, desc, false)) return r;
  p->exec_ready = true;
  p->ws_cap = want;
  p->part_cap = part;
  p->tri_cap = tri;
  return LIBPT_OK;
}

GemmGroup plan_group(const libpt_plan *p, const SpinCase &c) {
  GemmGroup g;
  if (p->precision == LIBPT_PREC_EMU64) {
    g.kind = 2;
    g.bm = TC_BM;
    g.slices = p->slices;
    g.tile = p->i8tile;
  } else if (p->precision == LIBPT_PREC_TF32X3) {
    g.kind = 1;
    g.bm = TC_BM;
  } else {
    g.kind = 0;
    g.bm = c.bm;
  }
  return g;
}

int plan_append(libpt_plan *p, const int64_t *ents, size_t n, PlanCursor &cur,
                Round &r, size_t *taken) {
  *taken = 0;
  const bool tc = p->precision == LIBPT_PREC_TF32X3;
  const bool i8 = p->precision == LIBPT_PREC_EMU64;
  for (size_t t = 0; t < n; ++t) {
    const int4 q = p->queue[ents[t]];
    SpinCase &c = p->cases[q.x];
    const int64_t wend = cur.ws_end >= 0 ? cur.ws_end : p->ws_cap;
    const int64_t pend = cur.part_end >= 0 ? cur.part_end : p->part_cap;
    const size_t tend = cur.tri_end ? cur.tri_end : p->tri_cap;
    if (cur.triples >= tend || cur.ws + c.ws_stride > wend ||
        cur.part + c.ntiles > pend)
      break;   // the round is full for this plan
    const int ijk[3] = {q.y, q.z, q.w};
    double *ws = p->ws + cur.ws;
    double *partials = p->partials + cur.part;
    cur.ws += c.ws_stride;
    cur.part += c.ntiles;
    ++cur.triples;
    ++*taken;
    const GemmGroup grp = plan_group(p, c);
    std::vector<GemmJob> &jobs = r.gemm[grp];
    const CUtensorMap *hmaps = p->precision == LIBPT_PREC_FP64 ? c.maps.m
                                                               : c.tcmaps.m;
    const int map0 = r.maps[grp].add(c.d_maps, hmaps, tc ? TC_MAX_MAPS : MAX_MAPS);
    const int bn = tc ? TC_BN : i8 ? p->i8tile.bn : GEMM_BN;
    const int bmr = tc ? TC_BM : i8 ? (p->i8tile.pair ? 2 : 1) * TC_BM : c.bm;
    for (const JobT &jt : c.jobs) {
      GemmJob g;
      memset(&g, 0, sizeof(g));
      g.out = ws + jt.off;
      g.ldc = jt.ldc;
      g.M = jt.M;
      g.N = jt.N;
      g.ea = jt.ea;
      g.eb = jt.eb;
      g.maps = c.d_maps;
      g.map0 = map0;
      g.dbits = i8 ? p->dbits : 0;
      g.ntiles_n = (jt.N + bn - 1) / bn;
      g.mtiles = (jt.M + bmr - 1) / bmr;
      g.nseg = jt.nseg;
      for (int s = 0; s < jt.nseg; ++s) {
        const SegT &st = jt.seg[s];
        GemmSeg &gs = g.seg[s];
        gs.amap = (int16_t)(tc ? 2 * st.amap : st.amap);
        gs.bmap = (int16_t)(tc ? 2 * st.bmap : st.bmap);
        // INT8: a subtracted segment reads the negated digit planes, stored
        // after the slices_store digit planes
        gs.neg = (int16_t)(st.neg ? (i8 ? p->slices_store : 1) : 0);
        gs.a_q = ijk[st.aq];
        gs.a_p = ijk[st.ap];
        if (i8) {   // INT8 A views merge (Q, P) into one coordinate
          gs.a_q = gs.a_p * (int32_t)c.opd[st.amap].Q + gs.a_q;
          gs.a_p = 0;
        }
        gs.b_p = ijk[st.bp];
        gs.ksteps = tc ? (st.k + tc_kchunk_elems(TC_TF32) - 1) /
                             tc_kchunk_elems(TC_TF32)
                  : i8 ? (st.k + p->i8tile.kc - 1) / p->i8tile.kc
                       : st.ksteps;
        gs.half_last = (int16_t)(i8 && st.k % p->i8tile.kc != 0 &&
                                 st.k % p->i8tile.kc <= 32);
      }
      jobs.push_back(g);
    }
    EpiItem e;
    memset(&e, 0, sizeof(e));
    e.args = c.d_epi;
    e.ws = ws;
    e.partials = partials;
    e.i = q.y;
    e.j = q.z;
    e.k = q.w;
    r.epi[c.type][p->ft ? 1 : 0].push_back(e);
    r.epi_blocks[c.type][p->ft ? 1 : 0].push_back(c.ntiles);
    if (p->has_f) r.epi_hasf[c.type][p->ft ? 1 : 0] = true;
    RedItem red;
    red.partials = e.partials;
    red.dst = p->e_slot + ents[t];
    red.n = c.ntiles;
    red.pad_ = 0;
    r.red.push_back(red);
    r.gemm_flops += c.flops_per_triple;
    ++r.triples;
  }
  return LIBPT_OK;
}

// Runs queue entries in rounds, each filling the plan's round resources.
int run_entries(libpt_plan *p, const std::vector<int64_t> &ents) {
  if (ents.empty()) return LIBPT_OK;
  if (int r = ensure_capacity(p, ents)) return r;
  Round round;
  for (size_t b0 = 0; b0 < ents.size();) {
    round.clear();
    PlanCursor cur;
    size_t taken = 0;
    if (int r = plan_append(p, ents.data() + b0, ents.size() - b0, cur, round,
                            &taken))
      return r;
    if (taken == 0) {
      set_error("a triple does not fit the round resources");
      return LIBPT_ERR_NOMEM;
    }
    b0 += taken;
    if (int r = p->exec.run(round, p->d_err, p->timing ? &p->tm : nullptr,
                            &p->launches))
      return r;
  }
  return LIBPT_OK;
}

int plan_run(libpt_plan *p, const int64_t *idx, size_t n) {
  if (!p->deferred.empty())
    if (int r = flush_deferred(p)) return r;
  const int64_t total = (int64_t)p->queue.size();
  std::vector<int64_t> ents(n);
  for (size_t x = 0; x < n; ++x) {
    const int64_t q = idx ? idx[x] : (int64_t)x;
    if (q < 0 || q >= total) {
      set_error("libpt_plan_run: queue index out of range");
      return LIBPT_ERR_ARG;
    }
    ents[x] = q;
  }
  return run_entries(p, ents);
}

int plan_energy(libpt_plan *p, const int64_t *idx, size_t n, double *e,
                cudaStream_t rs) {
  const size_t total = p->queue.size();
  const cudaStream_t st = rs ? rs : p->st;
  // the energy readback buffer comes from the caller's allocation hook
  double *slots = static_cast<double *>(host_alloc((total + 1) * 8));
  if (!slots) {
    set_error("host allocation hook failed");
    return LIBPT_ERR_NOMEM;
  }
  struct Guard {
    double *q;
    ~Guard() { host_free(q); }
  } guard{slots};
  CK(cudaMemcpyAsync(slots, p->e_slot, (total + 1) * 8,
                     cudaMemcpyDeviceToHost, st));
  unsigned err = 0;
  CK(cudaMemcpyAsync(&err, p->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                     st));
  CK(cudaStreamSynchronize(st));
  if (err) {
    set_error("a device-side wait exceeded its time limit");
    return LIBPT_ERR_TIMEOUT;
  }
  double s = 0.0;
  if (int r = sum_slots(slots, total, idx, n, &s)) return r;
  *e = p->factor * s;
  return LIBPT_OK;
}

double wall_seconds() {
  timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

bool profile_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("LIBPT_PROFILE");
    return e && e[0] == '1';
  }();
  return on;
}

int sum_slots(const double *slots, size_t total, const int64_t *idx, size_t n,
              double *out) {
  // Neumaier-compensated sum in queue order
  double s = 0.0, comp = 0.0;
  const size_t m = idx ? n : total;
  for (size_t x = 0; x < m; ++x) {
    const int64_t q = idx ? idx[x] : (int64_t)x;
    if (q < 0 || (size_t)q >= total) {
      set_error("energy sum: queue index out of range");
      return LIBPT_ERR_ARG;
    }
    const double v = slots[q];
    const double t = s + v;
    comp += std::fabs(s) >= std::fabs(v) ? (s - t) + v : (v - t) + s;
    s = t;
  }
  *out = s + comp;
  return LIBPT_OK;
}

int64_t shard_entries(int64_t total, int rank, int size, int64_t *idx) {
  // src/pt.c:213: triple `it` belongs to rank it % size
  if (total < 0 || size < 1 || rank < 0 || rank >= size) return -1;
  int64_t n = 0;
  for (int64_t q = rank; q < total; q += size) {
    if (idx) idx[n] = q;
    ++n;
  }
  return n;
}

int plan_run_shard(libpt_plan *p, int rank, int size) {
  const int64_t total = (int64_t)p->queue.size();
  const int64_t n = shard_entries(total, rank, size, nullptr);
  if (n < 0) {
    set_error("libpt_plan_run_shard: rank outside [0, size)");
    return LIBPT_ERR_ARG;
  }
  // every slot this rank does not own stays zero, so that summing the ranks'
  // slot arrays leaves each triple's energy exactly as its owner computed it
  CK(cudaMemsetAsync(p->e_slot, 0, (total + 1) * 8, p->st));
  std::vector<int64_t> ents((size_t)n);
  shard_entries(total, rank, size, ents.data());
  return run_entries(p, ents);
}

}  // namespace ptb
