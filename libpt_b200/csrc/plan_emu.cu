// Emulated FP64 operands: scale families, per-row / per-column maxima and
// power-of-two exponents, INT8 digit planes, the digit width and the slice
// count chosen for a stated tolerance.
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

Family *family(libpt_plan *p, int id, int64_t n) {
  for (Family &f : p->fams)
    if (f.id == id) return &f;
  Family f;
  f.id = id;
  f.n = n;
  if (dalloc(p, (void **)&f.max0, n * 8 + 8) ||
      dalloc(p, (void **)&f.max1, n * 8 + 8) || dalloc(p, (void **)&f.e, n + 16))
    return nullptr;
  if (!g_dry) {
    cudaMemsetAsync(f.max0, 0, n * 8 + 8, p->st);
    cudaMemsetAsync(f.max1, 0, n * 8 + 8, p->st);
  }
  p->fams.push_back(f);
  return &p->fams.back();
}

// Emulated FP64, phase 1: per-row / per-column maxima of every operand of
// every case, into its family's part (each operand once).
int i8_maxima(libpt_plan *p) {
  std::vector<std::pair<const double *, int>> seen;
  for (SpinCase &c : p->cases) {
    if (c.count == 0) continue;
    for (int i = 0; i < MAX_MAPS; ++i) {
      const OpDesc &d = c.opd[i];
      if (d.role < 0) continue;
      Family *f = family(p, d.fam, d.role == 0 ? d.R : d.N);
      if (!f) return LIBPT_ERR_NOMEM;
      const std::pair<const double *, int> key(d.src, d.role * 2 + d.part);
      if (std::find(seen.begin(), seen.end(), key) != seen.end()) continue;
      seen.push_back(key);
      unsigned long long *m = d.part ? f->max1 : f->max0;
      if (d.role == 0)
        DEV(rowmax_launch(d.src, d.P * d.Q, d.R, d.K, pad4(d.K), m, p->st));
      else
        DEV(colmax_launch(d.src, d.P, d.K, d.N, d.w, d.wsrc, d.ldsrc, m, p->st));
    }
  }
  return LIBPT_OK;
}

// Phase 2: per operand set, the power-of-two exchange between the OOVO and
// the amplitude operand sides that balances their magnitudes; phase 3: the
// joint exponents of every family.
int i8_exponents(libpt_plan *p) {
  std::vector<unsigned long long> h;
  for (int x = 0; x < (p->ft ? 2 : 1); ++x) {
    double m0 = 0.0, m1 = 0.0;
    for (Family &f : p->fams) {
      if (f.id >= 100 || f.id / 8 != x) continue;   // A families of set x
      for (int part = 0; part < 2; ++part) {
        h.assign(f.n, 0);
        DEV(cudaMemcpyAsync(h.data(), part ? f.max1 : f.max0, f.n * 8,
                            cudaMemcpyDeviceToHost, p->st));
        DEV(cudaStreamSynchronize(p->st));
        for (unsigned long long u : h) {
          double v;
          memcpy(&v, &u, 8);
          (part ? m1 : m0) = std::max(part ? m1 : m0, v);
        }
      }
    }
    OperandSet &S = x ? p->R : p->L;
    S.balance = (m0 > 0 && m1 > 0) ? (int)std::lround(std::log2(m1 / m0)) : 0;
  }
  for (Family &f : p->fams) {
    const int set = (f.id % 100) / 8;
    const int k = (set ? p->R : p->L).balance;
    const double s1 = std::ldexp(1.0, f.id >= 100 ? k : -k);
    DEV(exps_launch(f.max0, f.max1, s1, f.n, f.e, p->st));
  }
  return LIBPT_OK;
}

// Phase 4: digit planes of every operand and the INT8 tensor-core views.
// Tensor maps of a case's digit planes for the plan's current tile variant.
int i8_encode(libpt_plan *p, SpinCase &c) {
  for (int i = 0; i < MAX_MAPS; ++i) {
    const OpDesc &d = c.opd[i];
    if (d.role < 0) continue;
    const int r =
        d.role == 0
            ? i8_map_a(&c.tcmaps.m[i], c.i8pl[i], d.K, d.R, d.Q, d.P,
                       p->slices_store)
            : i8_map_b(&c.tcmaps.m[i], c.i8pl[i], d.K, d.N, d.P,
                       p->slices_store,
                       // a CTA of a pair tile loads half of its columns
                       p->i8tile.pair ? p->i8tile.bn / 2 : p->i8tile.bn);
    if (r) return r;
  }
  return LIBPT_OK;
}

// Digit planes of a case's operands (shared between cases by source).
int i8_planes(libpt_plan *p, SpinCase &c) {
  const int S = p->slices_store;
  for (int i = 0; i < MAX_MAPS; ++i) {
    const OpDesc &d = c.opd[i];
    if (d.role < 0) continue;
    Family *f = family(p, d.fam, d.role == 0 ? d.R : d.N);
    if (!f) return LIBPT_ERR_NOMEM;
    const int set = (d.fam % 100) / 8;
    const int k = (set ? p->R : p->L).balance;
    const int64_t kpi = i8_kpad(d.K);
    const std::pair<const double *, int> key(d.src, d.role);
    signed char *pl = nullptr;
    for (auto &e : p->i8planes)
      if (e.first == key) pl = e.second;
    if (!pl) {
      const int64_t n = d.role == 0 ? d.P * d.Q * d.R * kpi : d.P * d.N * kpi;
      if (dalloc(p, (void **)&pl, (d.role == 0 ? 2 : 1) * S * n))
        return LIBPT_ERR_NOMEM;
      p->i8planes.push_back({key, pl});
      if (d.role == 0)
        DEV(slice_a_launch(d.src, d.P * d.Q, d.R, d.K, pad4(d.K), kpi,
                          std::ldexp(1.0, d.part ? -k : 0), f->e, S, p->dbits,
                          pl, p->st));
      else
        DEV(slice_b_launch(d.src, d.P, (int)d.K, d.N, d.w, d.wsrc, d.ldsrc, kpi,
                          std::ldexp(1.0, d.part ? k : 0), f->e, S, p->dbits,
                          pl, p->st));
    }
    c.i8pl[i] = pl;
  }
  if (int r = i8_encode(p, c)) return r;
  // each job's output rows / columns take the scales of its operand families
  for (JobT &j : c.jobs) {
    for (Family &f : p->fams) {
      if (f.id == c.opd[j.seg[0].amap].fam) j.ea = f.e;
      if (f.id == c.opd[j.seg[0].bmap].fam) j.eb = f.e;
    }
  }
  return LIBPT_OK;
}

// Digit width of the INT8 planes.  Every accumulator (one digit-weight
// diagonal: at most S digit products per unit of K, summed over a job's
// segments) must stay below 2^31: S * 64^2 per unit of K for 7-bit digits,
// S * 128^2 for 8-bit ones.  8-bit digits (8 bits of the operand per lower
// plane instead of 7) are used for S <= 6 whenever they fit, unless
// LIBPT_EMU_DIGITS=7; a plan that chooses S itself then stores 6 planes
// (47 bits, about as accurate as 7 planes of 7 bits).
int choose_digits(libpt_plan *p) {
  int64_t kmax = 0;
  for (const SpinCase &c : p->cases)
    for (const JobT &j : c.jobs) {
      int64_t k = 0;
      for (int s = 0; s < j.nseg; ++s) k += j.seg[s].k;
      kmax = std::max(kmax, k);
    }
  const char *env = std::getenv("LIBPT_EMU_DIGITS");
  const bool allow8 = !(env && std::atoi(env) == 7);
  auto fits8 = [&](int S) {
    return allow8 && S <= 6 && (double)kmax * S * 16384.0 < 2147483648.0;
  };
  if (p->slices_auto) {
    const int S = fits8(6) ? 6 : TC_S_MAX;
    p->dbits = S == 6 ? 8 : 7;
    p->slices = p->slices_store = S;
    const I8Tile *t = nullptr;
    if (i8_tiles(S, &t) > 0) p->i8tile = t[0];
  } else {
    p->dbits = fits8(p->slices_store) ? 8 : 7;
  }
  if (p->dbits == 7 &&
      (double)kmax * 4096.0 * p->slices_store >= 2147483648.0) {
    set_error("emulated FP64: contraction too long for exact INT32 "
              "accumulation");
    return LIBPT_ERR_UNSUPPORTED;
  }
  return LIBPT_OK;
}

// Emulated FP64 with the slice count left to the library: the digit planes
// are built with the most slices (6 of 8 bits, or 7 of 7 bits; see
// choose_digits) and any S below runs on their first S planes, which are
// the S-digit decomposition (with 8-bit digits, but for rare carries into
// the last kept digit, which stay within the same error bound).
//
// Error model.  Digits are rounded to nearest, so the dropped digit products
// of a contraction element are zero-mean and their signs vary from element
// to element; the first-order energy error of a triple, sum (2W - V) dW / D,
// is then zero-mean, and triples (different amplitude rows) err
// independently.  The solve's error with S slices is therefore a sum of N
// independent per-triple errors: about sqrt(N) * rms(e_S - e_7) (the second-
// order term sum dW^2 / D is of relative size (dW/W)^2, below 1e-18 for
// S >= 4).  A sample of n = min(N, 16) triples spread over the queue is
// evaluated with all stored planes (e_max) and with S; the smallest S with
//     3 sqrt(N) rms_sample(e_S - e_max) * factor <= LIBPT_EMU_TOL / 2
// (default tolerance 1e-6 Eh) is kept.  LIBPT_EMU_BOUND=worst replaces the
// estimate by the cancellation-free bound (N / n) sum_sample |e_S - e_max|.
// Sampling costs about 3n triples; a solve with fewer than 40n triples
// (where that would exceed ~8 % of the solve) keeps all stored planes.
int choose_slices(libpt_plan *p) {
  const size_t N = p->queue.size();
  if (!N) return LIBPT_OK;
  const size_t n = std::min<size_t>(N, 16);
  const char *bound_env = std::getenv("LIBPT_EMU_BOUND");
  const bool worst = bound_env && std::strcmp(bound_env, "worst") == 0;
  auto apply = [&](int S) -> int {
    const I8Tile *tiles = nullptr;
    if (i8_tiles(S, &tiles) <= 0) return LIBPT_ERR_ARG;
    p->slices = S;
    p->i8tile = tiles[0];
    for (SpinCase &c : p->cases)
      if (c.count)
        if (int r = i8_encode(p, c)) return r;
    return upload_views(p);
  };
  const int smax = p->slices_store;   // 6 (8-bit digits) or 7 (7-bit)
  int chosen = smax;
  if (N >= 40 * n) {
    std::vector<int64_t> ents(n);
    for (size_t t = 0; t < n; ++t) ents[t] = (int64_t)(t * N / n);
    std::vector<double> slots(N + 1), ref(n);
    auto run_with = [&](int S, std::vector<double> &out) -> int {
      if (int r = apply(S)) return r;
      if (int r = run_entries(p, ents)) return r;
      CK(cudaMemcpyAsync(slots.data(), p->e_slot, (N + 1) * 8,
                         cudaMemcpyDeviceToHost, p->st));
      CK(cudaStreamSynchronize(p->st));
      out.resize(n);
      for (size_t t = 0; t < n; ++t) out[t] = slots[(size_t)ents[t]];
      return LIBPT_OK;
    };
    auto estimate = [&](const std::vector<double> &e) {
      double sum_abs = 0.0, sum_sq = 0.0;
      for (size_t t = 0; t < n; ++t) {
        const double d = e[t] - ref[t];
        sum_abs += std::fabs(d);
        sum_sq += d * d;
      }
      return p->factor * (worst ? sum_abs * (double)N / (double)n
                                : 3.0 * std::sqrt((double)N * sum_sq / (double)n));
    };
    if (int r = run_with(smax, ref)) return r;
    // try 5 first, then 4 (if 5 passed) or 6 (if not, and 6 < smax)
    std::vector<double> e;
    auto passes = [&](int S, bool *ok) -> int {
      if (int r = run_with(S, e)) return r;
      const double est = estimate(e);
      if (tune_verbose())
        std::fprintf(stderr, "libpt slices: S=%d error estimate %.3e Eh "
                             "(%s; target %.1e)\n", S, est,
                     worst ? "cancellation-free bound" : "3 sqrt(N) rms",
                     p->emu_tol);
      *ok = est <= 0.5 * p->emu_tol;
      return LIBPT_OK;
    };
    bool ok = false;
    if (int r = passes(5, &ok)) return r;
    if (ok) {
      chosen = 5;
      if (int r = passes(4, &ok)) return r;
      if (ok) chosen = 4;
    } else if (smax > 6) {
      if (int r = passes(6, &ok)) return r;
      if (ok) chosen = 6;
    }
  } else if (tune_verbose()) {
    std::fprintf(stderr, "libpt slices: %zu triples, too few to sample: %d\n",
                 N, smax);
  }
  if (int r = apply(chosen)) return r;
  CK(cudaMemsetAsync(p->e_slot, 0, (N + 1) * 8, p->st));
  CK(cudaStreamSynchronize(p->st));
  p->launches = 0;
  return LIBPT_OK;
}

}  // namespace ptb
