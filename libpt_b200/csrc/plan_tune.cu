// The autotuner: kernel variants of a plan chosen by timing them on a probe
// of its triples, remembered per (kind, sizes, precision, slices, dtype).
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

// Device time of one run of `ents` (of case c), in milliseconds.
int probe_ms(libpt_plan *p, SpinCase &c, const std::vector<int64_t> &ents,
             float *ms) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int r = LIBPT_OK;
  CK(cudaEventRecord(e0, p->st));
  r = run_entries(p, ents);
  if (!r) {
    CK(cudaEventRecord(e1, p->st));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return r;
}

// Re-encodes a case's DMMA A views for CTA tile rows bm.
int set_bm(SpinCase &c, int bm) {
  c.bm = bm;
  for (int i = 0; i < MAX_MAPS; ++i) {
    const OpDesc &d = c.opd[i];
    if (d.role == 0)
      if (int r = map_a(&c.maps.m[i], d.src, d.K, d.R, d.Q, d.P, bm)) return r;
  }
  return LIBPT_OK;
}

// The autotuner: picks the kernel variants of a plan by timing them on a
// probe of its triples (each candidate run twice, the second run timed),
// and remembers the choice per (kind, sizes, precision, slices, dtype).
//   FP64 DMMA:      CTA tile rows 96 or 128, per spin case
//   emulated FP64:  the INT8 tile variants of the slice count (i8_tiles)
// The probe's energies are discarded (slots reset afterwards); choices do
// not change results, only speed (each output element is accumulated in
// the same order by every variant).
// Sum over the spin cases of the autotuner's probe work (two timed runs per
// candidate on up to four triples of each case; emulated FP64: of the case
// with the most work).
double probe_flops(const libpt_plan *p, int ntiles) {
  const bool emu = p->precision == LIBPT_PREC_EMU64;
  double probe = 0.0;
  for (const SpinCase &c : p->cases)
    probe = emu ? std::max(probe, 2.0 * ntiles *
                                      (double)std::min<int64_t>(c.count, 4) *
                                      c.flops_per_triple)
                : probe + 4.0 * (double)std::min<int64_t>(c.count, 4) *
                              c.flops_per_triple;
  return probe;
}

// Whether plan creation will run autotuning probes (which read operands).
bool tune_would_probe(libpt_plan *p) {
  if (p->queue.empty() || p->precision == LIBPT_PREC_TF32X3 || g_dry)
    return false;
  const bool emu = p->precision == LIBPT_PREC_EMU64;
  const std::string key = tune_key(p->kind, p->oa, p->va, p->ob, p->vb,
                                   p->precision, emu ? p->slices : 0, p->dtype);
  std::vector<int> choice;
  if (tune_lookup(key, &choice) || !tune_enabled()) return false;
  const I8Tile *tiles = nullptr;
  const int ntiles = emu ? i8_tiles(p->slices, &tiles) : 0;
  return probe_flops(p, ntiles) <=
         0.05 * plan_flops(p, 0, (int64_t)p->queue.size());
}

int autotune(libpt_plan *p) {
  if (p->queue.empty() || p->precision == LIBPT_PREC_TF32X3) return LIBPT_OK;
  const bool emu = p->precision == LIBPT_PREC_EMU64;
  const std::string key = tune_key(p->kind, p->oa, p->va, p->ob, p->vb,
                                   p->precision, emu ? p->slices : 0, p->dtype);
  const I8Tile *tiles = nullptr;
  const int ntiles = emu ? i8_tiles(p->slices, &tiles) : 0;
  std::vector<int> choice;
  if (tune_lookup(key, &choice)) {
    if (emu && !choice.empty() && choice[0] >= 0 && choice[0] < ntiles) {
      p->i8tile = tiles[choice[0]];
      for (SpinCase &c : p->cases)
        if (c.count)
          if (int r = i8_encode(p, c)) return r;
    } else if (!emu && choice.size() == p->cases.size()) {
      for (size_t ci = 0; ci < p->cases.size(); ++ci)
        if (p->cases[ci].count && (choice[ci] == 96 || choice[ci] == 128))
          if (int r = set_bm(p->cases[ci], choice[ci])) return r;
    }
    return upload_views(p);
  }
  if (!tune_enabled()) return LIBPT_OK;
  // probe: the first triples of the case with the most work
  auto probe_of = [&](const SpinCase &c) {
    const int64_t n = std::min<int64_t>(c.count, 4);
    std::vector<int64_t> e((size_t)n);
    for (int64_t x = 0; x < n; ++x) e[(size_t)x] = c.first + x;
    return e;
  };
  {
    // a small solve keeps the defaults: its probes (two timed runs per
    // candidate) would cost more than a better tile could save
    const double probe = probe_flops(p, ntiles);
    if (probe > 0.05 * plan_flops(p, 0, (int64_t)p->queue.size())) {
      if (tune_verbose())
        std::fprintf(stderr, "libpt autotune %s: skipped (probes %.3g flops "
                             "> 5%% of the solve)\n", key.c_str(), probe);
      return LIBPT_OK;
    }
  }
  int r = LIBPT_OK;
  if (emu) {
    size_t big = 0;
    double most = -1.0;
    for (size_t ci = 0; ci < p->cases.size(); ++ci) {
      const SpinCase &c = p->cases[ci];
      const double w = (double)c.count * c.flops_per_triple;
      if (c.count && w > most) {
        most = w;
        big = ci;
      }
    }
    const std::vector<int64_t> ents = probe_of(p->cases[big]);
    int best = 0;
    float best_ms = 0.f;
    for (int t = 0; t < ntiles && !r; ++t) {
      p->i8tile = tiles[t];
      r = i8_encode(p, p->cases[big]);
      if (!r) r = upload_views(p);
      float ms = 0.f;
      if (!r) r = probe_ms(p, p->cases[big], ents, &ms);
      if (!r) r = probe_ms(p, p->cases[big], ents, &ms);
      if (!r && tune_verbose())
        std::fprintf(stderr, "libpt autotune %s: INT8 tile %dx%d, K chunk %d B: %.3f ms\n",
                     key.c_str(), (tiles[t].pair ? 2 : 1) * TC_BM, tiles[t].bn,
                     tiles[t].kc, ms);
      if (!r && (t == 0 || ms < best_ms)) {
        best = t;
        best_ms = ms;
      }
    }
    if (r) return r;
    p->i8tile = tiles[best];
    for (SpinCase &c : p->cases)
      if (c.count)
        if ((r = i8_encode(p, c))) return r;
    if ((r = upload_views(p))) return r;
    choice.assign(1, best);
  } else {
    choice.assign(p->cases.size(), 0);
    for (size_t ci = 0; ci < p->cases.size() && !r; ++ci) {
      SpinCase &c = p->cases[ci];
      if (!c.count) continue;
      const std::vector<int64_t> ents = probe_of(c);
      const int start = c.bm;
      int best = start;
      float best_ms = 0.f;
      for (int bm : {start, start == 96 ? 128 : 96}) {
        if ((r = set_bm(c, bm))) break;
        if ((r = upload_views(p))) break;
        float ms = 0.f;
        if ((r = probe_ms(p, c, ents, &ms))) break;
        if ((r = probe_ms(p, c, ents, &ms))) break;
        if (tune_verbose())
          std::fprintf(stderr, "libpt autotune %s: case %zu, DMMA tile rows %d: %.3f ms\n",
                       key.c_str(), ci, bm, ms);
        if (bm == start || ms < best_ms) {
          best = bm;
          best_ms = ms;
        }
      }
      if (!r) r = set_bm(c, best);
      if (!r) r = upload_views(p);
      choice[ci] = best;
    }
    if (r) return r;
  }
  tune_store(key, choice);
  p->launches = 0;
  // forget the probe's energies
  CK(cudaMemsetAsync(p->e_slot, 0, (p->queue.size() + 1) * 8, p->st));
  CK(cudaStreamSynchronize(p->st));
  return LIBPT_OK;
}

}  // namespace ptb
