// Spin cases and their per-triple job templates: the signed K segments of
// the same-spin (T) and mixed-spin (U1, U2, P) contractions, derived term by
// term from src/pt.c:236-290 and 361-432 (and their (fT) pairs,
// src/pt.c:588-696, 773-915), and the triples queue (src/pt.c:210-221,
// 333-344; spin cases in the order of src/pt.c:469-473, 514-529).
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

SegT seg(int amap, int bmap, bool neg, int aq, int ap, int bp, int64_t k) {
  SegT s;
  s.amap = (int16_t)amap;
  s.bmap = (int16_t)bmap;
  s.neg = neg ? 1 : 0;
  s.aq = (int8_t)aq;
  s.ap = (int8_t)ap;
  s.bp = (int8_t)bp;
  s.ksteps = ksteps(k);
  s.k = (int32_t)k;
  return s;
}

// Symbolic occupied indices of a segment (SegT::aq / ap / bp).
enum { I = 0, J = 1, K = 2 };

// Encode a DMMA view (FP64 path) and remember what it views, for the
// tensor-core paths; fam/part classify the operand for emulated FP64.
int reg_a(libpt_plan *p, SpinCase &c, int idx, const double *ptr, int64_t Kd,
          int64_t R, int64_t Q, int64_t P, int fam, int part) {
  OpDesc &d = c.opd[idx];
  d.role = 0;
  d.src = ptr;
  d.K = Kd;
  d.R = R;
  d.Q = Q;
  d.P = P;
  d.fam = fam;
  d.part = part;
  if (p->precision != LIBPT_PREC_FP64) return LIBPT_OK;
  return map_a(&c.maps.m[idx], ptr, Kd, R, Q, P, c.bm);
}

// B operand [P][K][N] in the engine's padded layout (row length Nld), or --
// when src_w > 0 -- the caller's unpadded pt.h block whose N index is
// row-padded: n = y*src_w + c, c < src_wsrc real, rows of src_ld elements.
int reg_b(libpt_plan *p, SpinCase &c, int idx, const double *ptr, int64_t N,
          int64_t Nld, int64_t Kd, int64_t P, int fam, int part,
          int64_t src_ld = 0, int64_t src_w = 0, int64_t src_wsrc = 0) {
  OpDesc &d = c.opd[idx];
  d.role = 1;
  d.src = ptr;
  d.K = Kd;
  d.N = N;
  d.Nld = Nld;
  d.P = P;
  d.fam = fam;
  d.part = part;
  if (src_w > 0) {
    d.ldsrc = src_ld;
    d.w = src_w;
    d.wsrc = src_wsrc;
  } else {
    d.ldsrc = Nld;
    d.w = Nld;
    d.wsrc = Nld;
  }
  if (p->precision != LIBPT_PREC_FP64) return LIBPT_OK;
  return map_b(&c.maps.m[idx], ptr, N, Nld, Kd, P);
}

// Scale families of emulated FP64: the A operands of a job (amplitude and
// OOVO blocks of one spin-block index) and its B operands (OVVV block and
// the amplitude block of the same index) share row / column scales.
int fam_a(const libpt_plan *p, int set, int b) {
  return set * 8 + (!p->unrestricted && b == 3 ? 1 : b);
}

int fam_b(const libpt_plan *p, int set, int b) {
  return 100 + set * 8 + (!p->unrestricted && b == 3 ? 1 : b);
}

// OVVV block b of a set as a B operand: the padded FP64 copy, or the
// caller's pt.h block when it is sliced in place (emulated FP64, device
// inputs).  N counts the padded-convention columns.
int reg_ovvv(libpt_plan *p, SpinCase &c, int idx, const OperandSet &S, int b,
             int64_t N, int64_t Nld, int64_t Kd, int64_t P, int fam) {
  if (S.ovvv[b])
    return reg_b(p, c, idx, S.ovvv[b], N, Nld, Kd, P, fam, 0);
  const int64_t va = p->va, vb = p->vb;
  int64_t ld, w, wsrc;
  if (b == 0 || b == 2) {   // packed pairs: no inner padding
    const int64_t v = b ? vb : va;
    ld = w = wsrc = v * (v - 1) / 2;
  } else if (b == 1) {      // [oa][vb][va][vb]: N = (y < va, c < vb)
    ld = va * vb;
    w = pad4(vb);
    wsrc = vb;
  } else {                  // [ob][va][vb][va]
    ld = vb * va;
    w = pad4(va);
    wsrc = va;
  }
  return reg_b(p, c, idx, S.ovvv_src[b], N, Nld, Kd, P, fam, 0, ld, w, wsrc);
}

// Same-spin case: four maps per operand set, one job (T) per set.
int build_aaa(libpt_plan *p, SpinCase &c) {
  const int s = c.flip;
  const int64_t o = c.oa, v = c.va, np = npair(v), ldT = pad4(np);
  const int nset = p->ft ? 2 : 1;
  int64_t offs[2];
  int64_t stride = 0;
  for (int x = 0; x < nset; ++x) {
    offs[x] = stride;
    stride += pad32(v * ldT);
  }
  for (int x = 0; x < nset; ++x) {
    const OperandSet &set = x ? p->R : p->L;
    const int b0 = 4 * x;
    const int bi = s ? 2 : 0;
    const int fa = fam_a(p, x, bi), fb = fam_b(p, x, bi);
    if (int r = reg_a(p, c, b0 + 0, set.tau[bi], v, v, o, o, fa, 0)) return r;
    if (int r = reg_a(p, c, b0 + 1, set.oovo[bi], o, v, o, o, fa, 1)) return r;
    if (int r = reg_ovvv(p, c, b0 + 2, set, bi, np, ldT, v, o, fb)) return r;
    if (int r = reg_b(p, c, b0 + 3, set.taup[s], np, ldT, o, o, fb, 1)) return r;
    JobT j;
    j.off = offs[x];
    j.M = (int)v;
    j.N = (int)ldT;
    j.ldc = ldT;
    j.nseg = 6;
    // T[x][pair] = sum_d (t_ij - t_ik - t_kj)[x][d] I_(k,j,i)[d][pair]
    //            + sum_l (O_jk - O_ik - O_ji)[x][l] tp_(i,j,k)[l][pair]
    j.seg[0] = seg(b0 + 0, b0 + 2, false, J, I, K, v);
    j.seg[1] = seg(b0 + 0, b0 + 2, true, K, I, J, v);
    j.seg[2] = seg(b0 + 0, b0 + 2, true, J, K, I, v);
    j.seg[3] = seg(b0 + 1, b0 + 3, false, K, J, I, o);
    j.seg[4] = seg(b0 + 1, b0 + 3, true, K, I, J, o);
    j.seg[5] = seg(b0 + 1, b0 + 3, true, I, J, K, o);
    if (np > 0) c.jobs.push_back(j);
  }
  EpiArgs &e = c.epi;
  memset(&e, 0, sizeof(e));
  c.ws_stride = stride;
  e.offL[0] = offs[0];
  e.offR[0] = p->ft ? offs[1] : -1;
  e.ld[0] = ldT;
  e.oa = (int)o;
  e.va = (int)v;
  e.ob = (int)o;
  e.vb = (int)v;
  const int64_t ovoff = s ? (int64_t)p->oa * p->va : 0;
  e.d_a = p->d_ov + ovoff;
  e.ov1_a = p->ov1 + ovoff;
  e.ov2_a = p->ov2 + ovoff;
  e.g1_aa = p->oovv[s ? 2 : 0];
  e.g1_ld_aa = v;
  e.g2_aa = p->L.tau[s ? 2 : 0];
  e.g2_ld_aa = pad4(v);
  // tiles (a0, b0, c0) holding at least one a > b > c
  std::vector<int4> tiles;
  for (int64_t a0 = 0; a0 < v; a0 += EPI_A) {
    const int64_t amax = std::min<int64_t>(a0 + EPI_A - 1, v - 1);
    for (int64_t b0 = 0; b0 <= a0; b0 += EPI_B) {
      if (amax - 1 < b0) continue;
      const int64_t bmax = std::min<int64_t>(b0 + EPI_B - 1, amax - 1);
      for (int64_t c0 = 0; c0 < bmax; c0 += EPI_C)
        tiles.push_back(make_int4((int)a0, (int)b0, (int)c0, 0));
    }
  }
  c.ntiles = (int)tiles.size();
  c.ctiles = 1;
  if (c.ntiles) {
    if (dalloc(p, (void **)&c.d_tiles, tiles.size() * sizeof(int4))) return LIBPT_ERR_NOMEM;
    DEV(cudaMemcpyAsync(c.d_tiles, tiles.data(), tiles.size() * sizeof(int4),
                       cudaMemcpyHostToDevice, p->st));
    DEV(cudaStreamSynchronize(p->st));
  }
  e.ntiles = c.ntiles;
  e.tiles = c.d_tiles;
  e.ctiles = c.ctiles;
  e.has_f = p->has_f ? 1 : 0;
  const double vv = (double)v;
  c.flops_per_triple = 3.0 * vv * vv * vv * (vv - 1) + 6.0 * o * vv * vv * vv;
  if (p->ft) c.flops_per_triple *= 2;
  return LIBPT_OK;
}

// Mixed-spin case: twelve maps per operand set, three jobs (U1, U2, P).
int build_aab(libpt_plan *p, SpinCase &c) {
  const int f = c.flip;
  const int64_t oa = c.oa, va = c.va, ob = c.ob, vb = c.vb;
  const int64_t np = npair(va);
  const int64_t ld1 = va * pad4(vb), ld2 = vb * pad4(va), ldP = pad4(np);
  const int nset = p->ft ? 2 : 1;
  int64_t offs[2][3];
  int64_t stride = 0;
  for (int x = 0; x < nset; ++x) {
    offs[x][0] = stride;
    stride += pad32(va * ld1);
    offs[x][1] = stride;
    stride += pad32(va * ld2);
    offs[x][2] = stride;
    stride += pad32(vb * ldP);
  }
  // block roles (src/pt.c:521-529): flip swaps alpha and beta
  const int Taa = f ? 2 : 0, Tab = f ? 3 : 1, Tba = f ? 1 : 3;
  for (int x = 0; x < nset; ++x) {
    const OperandSet &S = x ? p->R : p->L;
    const int m = 12 * x;
    int r;
    const int A0 = fam_a(p, x, Taa), A1 = fam_a(p, x, Tab),
              A3 = fam_a(p, x, Tba);
    const int B0 = fam_b(p, x, Taa), B1 = fam_b(p, x, Tab),
              B3 = fam_b(p, x, Tba);
    if ((r = reg_a(p, c, m + 0, S.tau[Taa], va, va, oa, oa, A0, 0))) return r;
    if ((r = reg_a(p, c, m + 1, S.tau[Tab], vb, va, ob, oa, A1, 0))) return r;
    if ((r = reg_a(p, c, m + 2, S.tau[Tba], va, vb, oa, ob, A3, 0))) return r;
    if ((r = reg_a(p, c, m + 3, S.oovo[Taa], oa, va, oa, oa, A0, 1))) return r;
    if ((r = reg_a(p, c, m + 4, S.oovo[Tab], ob, va, ob, oa, A1, 1))) return r;
    if ((r = reg_a(p, c, m + 5, S.oovo[Tba], oa, vb, oa, ob, A3, 1))) return r;
    if ((r = reg_ovvv(p, c, m + 6, S, Taa, np, ldP, va, oa, B0))) return r;
    if ((r = reg_ovvv(p, c, m + 7, S, Tab, ld1, ld1, vb, oa, B1))) return r;
    if ((r = reg_ovvv(p, c, m + 8, S, Tba, ld2, ld2, va, ob, B3))) return r;
    if ((r = reg_b(p, c, m + 9, S.taup[f], np, ldP, oa, oa, B0, 1))) return r;
    if ((r = reg_b(p, c, m + 10, S.tau[Tab], ld1, ld1, ob, oa, B1, 1))) return r;
    if ((r = reg_b(p, c, m + 11, S.tau[Tba], ld2, ld2, oa, ob, B3, 1))) return r;
    const int b = 12 * x;
    JobT u1, u2, pp;
    // U1[x][y,c] = -t_ik I_j + t_jk I_i + O_jk t_i - O_ik t_j
    u1.off = offs[x][0];
    u1.M = (int)va;
    u1.N = (int)ld1;
    u1.ldc = ld1;
    u1.nseg = 4;
    u1.seg[0] = seg(b + 1, b + 7, true, K, I, J, vb);
    u1.seg[1] = seg(b + 1, b + 7, false, K, J, I, vb);
    u1.seg[2] = seg(b + 4, b + 10, false, K, J, I, ob);
    u1.seg[3] = seg(b + 4, b + 10, true, K, I, J, ob);
    // U2[x][c,y] = -t_ij I_k + O_ji t_k
    u2.off = offs[x][1];
    u2.M = (int)va;
    u2.N = (int)ld2;
    u2.ldc = ld2;
    u2.nseg = 2;
    u2.seg[0] = seg(b + 0, b + 8, true, J, I, K, va);
    u2.seg[1] = seg(b + 3, b + 11, false, I, J, K, oa);
    // P[c][pair] = -t_kj I_i + t_ki I_j - O_kj tp_i + O_ki tp_j
    pp.off = offs[x][2];
    pp.M = (int)vb;
    pp.N = (int)ldP;
    pp.ldc = ldP;
    pp.nseg = 4;
    pp.seg[0] = seg(b + 2, b + 6, true, J, K, I, va);
    pp.seg[1] = seg(b + 2, b + 6, false, I, K, J, va);
    pp.seg[2] = seg(b + 5, b + 9, true, J, K, I, oa);
    pp.seg[3] = seg(b + 5, b + 9, false, I, K, J, oa);
    c.jobs.push_back(u1);
    c.jobs.push_back(u2);
    if (np > 0) c.jobs.push_back(pp);
  }
  EpiArgs &e = c.epi;
  memset(&e, 0, sizeof(e));
  c.ws_stride = stride;
  for (int q = 0; q < 3; ++q) {
    e.offL[q] = offs[0][q];
    e.offR[q] = p->ft ? offs[1][q] : -1;
  }
  e.ld[0] = ld1;
  e.ld[1] = ld2;
  e.ld[2] = ldP;
  e.rowU1 = pad4(vb);
  e.rowU2 = pad4(va);
  e.oa = (int)oa;
  e.va = (int)va;
  e.ob = (int)ob;
  e.vb = (int)vb;
  const int64_t offA = f ? (int64_t)p->oa * p->va : 0;
  const int64_t offB = f ? 0 : (int64_t)p->oa * p->va;
  const int64_t offB_r = p->unrestricted ? offB : 0;
  e.d_a = p->d_ov + offA;
  e.d_b = p->d_ov + offB_r;
  e.ov1_a = p->ov1 + offA;
  e.ov1_b = p->ov1 + offB_r;
  e.ov2_a = p->ov2 + offA;
  e.ov2_b = p->ov2 + offB_r;
  e.g1_ab = p->oovv[Tab];
  e.g1_ld_ab = vb;
  e.g1_aa = p->oovv[Taa];
  e.g1_ld_aa = va;
  e.g2_ab = p->L.tau[Tab];
  e.g2_ld_ab = pad4(vb);
  e.g2_aa = p->L.tau[Taa];
  e.g2_ld_aa = pad4(va);
  std::vector<int4> tiles;
  for (int64_t a0 = 0; a0 < va; a0 += EPI_A) {
    const int64_t amax = std::min<int64_t>(a0 + EPI_A - 1, va - 1);
    for (int64_t b0 = 0; b0 <= a0; b0 += EPI_B)
      if (amax - 1 >= b0) tiles.push_back(make_int4((int)a0, (int)b0, 0, 0));
  }
  c.ctiles = (int)((vb + EPI_C - 1) / EPI_C);
  c.ntiles = (int)tiles.size() * c.ctiles;
  if (!tiles.empty()) {
    if (dalloc(p, (void **)&c.d_tiles, tiles.size() * sizeof(int4))) return LIBPT_ERR_NOMEM;
    DEV(cudaMemcpyAsync(c.d_tiles, tiles.data(), tiles.size() * sizeof(int4),
                       cudaMemcpyHostToDevice, p->st));
    DEV(cudaStreamSynchronize(p->st));
  }
  e.ntiles = c.ntiles;
  e.tiles = c.d_tiles;
  e.ctiles = c.ctiles;
  e.has_f = p->has_f ? 1 : 0;
  const double A = (double)va, B = (double)vb;
  c.flops_per_triple = 2 * A * A * A * B + 4 * A * A * B * B +
                       2 * B * A * A * (A - 1) + 6 * A * A * B * oa +
                       4 * A * A * B * ob;
  if (p->ft) c.flops_per_triple *= 2;
  return LIBPT_OK;
}

int add_cases(libpt_plan *p) {
  const int oa = p->oa, va = p->va, ob = p->ob, vb = p->vb;
  auto add = [&](int type, int flip, int o1, int v1, int o2, int v2) {
    SpinCase c;
    c.type = type;
    c.flip = flip;
    c.oa = o1;
    c.va = v1;
    c.ob = o2;
    c.vb = v2;
    c.first = (int64_t)p->queue.size();
    const int ci = (int)p->cases.size();
    // src/pt.c:195-196, 318-319: an empty space contributes nothing
    const bool empty = type == 0 ? (o1 == 0 || v1 == 0)
                                 : (o1 == 0 || v1 == 0 || o2 == 0 || v2 == 0);
    if (!empty) {
      if (type == 0) {
        for (int i = 0; i < o1; ++i)
          for (int j = i + 1; j < o1; ++j)
            for (int k = j + 1; k < o1; ++k)
              p->queue.push_back(make_int4(ci, i, j, k));
      } else {
        for (int i = 0; i < o1; ++i)
          for (int j = i + 1; j < o1; ++j)
            for (int k = 0; k < o2; ++k)
              p->queue.push_back(make_int4(ci, i, j, k));
      }
    }
    c.count = (int64_t)p->queue.size() - c.first;
    p->cases.push_back(c);
  };
  add(0, 0, oa, va, oa, va);
  if (p->unrestricted) add(0, 1, ob, vb, ob, vb);
  add(1, 0, oa, va, ob, vb);
  if (p->unrestricted) add(1, 1, ob, vb, oa, va);
  for (SpinCase &c : p->cases) {
    if (c.count == 0) continue;
    // CTA tile rows: the choice that pads the GEMM rows (va, and vb for the
    // mixed-spin P job) least; ties go to 128 (more CTAs)
    auto padded = [](int64_t m, int64_t bm) { return (m + bm - 1) / bm * bm; };
    const int64_t w128 = padded(c.va, 128) + (c.type ? padded(c.vb, 128) : 0);
    const int64_t w96 = padded(c.va, 96) + (c.type ? padded(c.vb, 96) : 0);
    c.bm = w96 < w128 ? 96 : 128;
    int r = c.type == 0 ? build_aaa(p, c) : build_aab(p, c);
    if (!r && p->precision == LIBPT_PREC_TF32X3) r = build_tc(p, c);
    if (r) return r;
  }
  if (p->precision == LIBPT_PREC_EMU64) {
    if (int r = choose_digits(p)) return r;
    if (int r = i8_maxima(p)) return r;
    if (int r = i8_exponents(p)) return r;
    for (SpinCase &c : p->cases)
      if (c.count)
        if (int r = i8_planes(p, c)) return r;
  }
  return LIBPT_OK;
}

// Copies each case's kernel views (tensor maps) and epilogue arguments to
// device memory, where the kernels read them.  Re-run after any map change.
int upload_views(libpt_plan *p) {
  for (SpinCase &c : p->cases) {
    if (!c.count) continue;
    const size_t mb = sizeof(TcMapSet);   // >= sizeof(MapSet)
    if (!c.d_maps && dalloc(p, (void **)&c.d_maps, mb)) return LIBPT_ERR_NOMEM;
    if (!c.d_epi && dalloc(p, (void **)&c.d_epi, sizeof(EpiArgs)))
      return LIBPT_ERR_NOMEM;
    const void *src = p->precision == LIBPT_PREC_FP64
                          ? (const void *)&c.maps
                          : (const void *)&c.tcmaps;
    const size_t n = p->precision == LIBPT_PREC_FP64 ? sizeof(MapSet)
                                                     : sizeof(TcMapSet);
    DEV(cudaMemcpyAsync(c.d_maps, src, n, cudaMemcpyHostToDevice, p->st));
    DEV(cudaMemcpyAsync(c.d_epi, &c.epi, sizeof(EpiArgs),
                       cudaMemcpyHostToDevice, p->st));
  }
  // the sources are members of the plan, copied before they can change
  DEV(cudaStreamSynchronize(p->st));
  return LIBPT_OK;
}

}  // namespace ptb
