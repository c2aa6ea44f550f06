"""Seeded synthetic inputs in pt.h layout.

Distributions (one 64-bit seed per case):
  occupied orbital energies e_i ~ U[-1.5, -0.3], virtual e_a ~ U[0.1, 3.0],
  d_ov[i,a] = e_i - e_a  (plus omega/3 for (fT): the excitation shift omega ~
  U[0.2, 0.5] folded into the three denominator terms);
  t1, l1 ~ N(0, 1e-3); t2, l2 ~ N(0, 1e-2); i_oovv, i_ovvv, i_oovo and the
  (fT) intermediates ~ N(0, 5e-2) (standard deviations);
  f_ov = f2_ov = 0 unless `fock` is given (then N(0, fock)).
Symmetries, as pt.h requires:
  restricted: abab blocks with x[i,j,a,b] = x[j,i,b,a] (t2, l2, i_oovv);
  same-spin blocks derived from abab: t2_aaaa = t2_abab - t2_abab(a<->b),
  i_oovo_aaaa = i_oovo_abab - i_oovo_abab(i<->j), and the packed aaaa OVVV
  from the expanded abab block minus its (b<->c) transpose;
  unrestricted: same-spin blocks antisymmetrised in their own index pairs,
  baba amplitude/oovv blocks the transposes of abab (spin-orbital symmetry),
  other mixed blocks independent.
"""
import numpy as np


def _pack_pairs(x):
    """[..., v, v] antisymmetric -> [..., v(v-1)/2] over b>c, row-major."""
    v = x.shape[-1]
    r, c = np.tril_indices(v, -1)
    return np.ascontiguousarray(x[..., r, c])


def _antisym2(x, ax1, ax2):
    return x - np.swapaxes(x, ax1, ax2)


def _energies(rng, o, v):
    ei = rng.uniform(-1.5, -0.3, size=o)
    ea = rng.uniform(0.1, 3.0, size=v)
    return ei[:, None] - ea[None, :]


def _restricted_blocks(rng, o, v, amp):
    """(aaaa, abab) blocks of a t2-like tensor [o,o,v,v]."""
    x = rng.normal(0.0, amp, size=(o, o, v, v))
    ab = 0.5 * (x + x.transpose(1, 0, 3, 2))
    aa = ab - ab.transpose(0, 1, 3, 2)
    return aa, ab


def _oovo_restricted(rng, o, v, amp):
    ab = rng.normal(0.0, amp, size=(o, o, v, o))
    aa = ab - ab.transpose(1, 0, 2, 3)
    return aa, ab


def _ovvv_restricted(rng, o, v, amp):
    ab = rng.normal(0.0, amp, size=(o, v, v, v))
    aa = _pack_pairs(ab - ab.transpose(0, 1, 3, 2))
    return aa, ab


def _cat(*blocks):
    return np.concatenate([np.ascontiguousarray(b).ravel() for b in blocks])


def rpt_case(o, v, seed=0, fock=0.0):
    rng = np.random.default_rng(seed)
    t2aa, t2ab = _restricted_blocks(rng, o, v, 1e-2)
    gaa, gab = _restricted_blocks(rng, o, v, 5e-2)
    oaa, oab = _oovo_restricted(rng, o, v, 5e-2)
    vaa, vab = _ovvv_restricted(rng, o, v, 5e-2)
    return dict(kind="rpt", oa=o, va=v, ob=o, vb=v,
                d_ov=_energies(rng, o, v).ravel(),
                f_ov=(rng.normal(0.0, fock, size=o * v) if fock
                      else np.zeros(o * v)),
                t1=rng.normal(0.0, 1e-3, size=o * v),
                t2=_cat(t2aa, t2ab), i_oovo=_cat(oaa, oab),
                i_oovv=_cat(gaa, gab), i_ovvv=_cat(vaa, vab))


def _same_spin_oovv(rng, o, v, amp):
    x = rng.normal(0.0, amp, size=(o, o, v, v))
    return 0.5 * _antisym2(_antisym2(x, 0, 1), 2, 3)


def _ovvv_same(rng, o, v, amp):
    x = rng.normal(0.0, amp, size=(o, v, v, v))
    return _pack_pairs(_antisym2(x, 2, 3))


def upt_case(oa, va, ob, vb, seed=0, fock=0.0):
    rng = np.random.default_rng(seed)

    def oovv_like(amp):
        aa = _same_spin_oovv(rng, oa, va, amp)
        ab = rng.normal(0.0, amp, size=(oa, ob, va, vb))
        bb = _same_spin_oovv(rng, ob, vb, amp)
        ba = ab.transpose(1, 0, 3, 2)
        return _cat(aa, ab, bb, ba)

    def oovo_like(amp):
        aa = _antisym2(rng.normal(0.0, amp, size=(oa, oa, va, oa)), 0, 1)
        ab = rng.normal(0.0, amp, size=(oa, ob, va, ob))
        bb = _antisym2(rng.normal(0.0, amp, size=(ob, ob, vb, ob)), 0, 1)
        ba = rng.normal(0.0, amp, size=(ob, oa, vb, oa))
        return _cat(aa, ab, bb, ba)

    def ovvv_like(amp):
        aa = _ovvv_same(rng, oa, va, amp)
        ab = rng.normal(0.0, amp, size=(oa, vb, va, vb))
        bb = _ovvv_same(rng, ob, vb, amp)
        ba = rng.normal(0.0, amp, size=(ob, va, vb, va))
        return _cat(aa, ab, bb, ba)

    d = _cat(_energies(rng, oa, va), _energies(rng, ob, vb))
    nov = oa * va + ob * vb
    return dict(kind="upt", oa=oa, va=va, ob=ob, vb=vb, d_ov=d,
                f_ov=rng.normal(0.0, fock, size=nov) if fock else np.zeros(nov),
                t1=rng.normal(0.0, 1e-3, size=nov),
                t2=oovv_like(1e-2), i_oovo=oovo_like(5e-2),
                i_oovv=oovv_like(5e-2), i_ovvv=ovvv_like(5e-2))


def rft_case(o, v, seed=0, fock=0.0):
    rng = np.random.default_rng(seed)
    omega = rng.uniform(0.2, 0.5)
    t2aa, t2ab = _restricted_blocks(rng, o, v, 1e-2)
    l2aa, l2ab = _restricted_blocks(rng, o, v, 1e-2)
    gaa, gab = _restricted_blocks(rng, o, v, 5e-2)
    i2 = _oovo_restricted(rng, o, v, 5e-2)
    i6 = _oovo_restricted(rng, o, v, 5e-2)
    i3 = _ovvv_restricted(rng, o, v, 5e-2)
    i7 = _ovvv_restricted(rng, o, v, 5e-2)
    return dict(kind="rft", oa=o, va=v, ob=o, vb=v, omega=omega,
                d_ov=_energies(rng, o, v).ravel() + omega / 3.0,
                f2_ov=(rng.normal(0.0, fock, size=o * v) if fock
                       else np.zeros(o * v)),
                l1=rng.normal(0.0, 1e-3, size=o * v),
                t2=_cat(t2aa, t2ab), l2=_cat(l2aa, l2ab),
                i_oovv=_cat(gaa, gab), i2_t2f2_oovo=_cat(*i2),
                i3_ovvv=_cat(*i3), i6_oovo=_cat(*i6), i7_ovvv=_cat(*i7))


def uft_case(oa, va, ob, vb, seed=0, fock=0.0):
    base = upt_case(oa, va, ob, vb, seed=seed, fock=fock)
    rng = np.random.default_rng(seed + 0x5eed)
    omega = rng.uniform(0.2, 0.5)
    other = [upt_case(oa, va, ob, vb, seed=seed + 1 + s) for s in range(3)]
    return dict(kind="uft", oa=oa, va=va, ob=ob, vb=vb, omega=omega,
                d_ov=base["d_ov"] + omega / 3.0, f2_ov=base["f_ov"],
                l1=base["t1"], t2=base["t2"], l2=other[0]["t2"],
                i_oovv=base["i_oovv"], i2_t2f2_oovo=base["i_oovo"],
                i3_ovvv=base["i_ovvv"], i6_oovo=other[1]["i_oovo"],
                i7_ovvv=other[2]["i_ovvv"])


def make(kind, oa, va, ob=None, vb=None, seed=0, fock=0.0):
    if kind == "rpt":
        return rpt_case(oa, va, seed, fock)
    if kind == "rft":
        return rft_case(oa, va, seed, fock)
    ob = oa if ob is None else ob
    vb = va if vb is None else vb
    if kind == "upt":
        return upt_case(oa, va, ob, vb, seed, fock)
    if kind == "uft":
        return uft_case(oa, va, ob, vb, seed, fock)
    raise ValueError(kind)


def rpt_case_device(o, v, seed=0, device="cuda", fock=0.0):
    """Restricted (T) inputs generated on the GPU with torch, block by block,
    for shapes too large for host generation (o=45, v=477 holds 74 GB).
    Same distributions and symmetries as rpt_case (not the same numbers).
    Returns (meta, tensors) with pt.h-layout float64 CUDA tensors."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    f64 = dict(dtype=torch.float64, device=device)

    def normal(shape, std):
        return torch.randn(shape, generator=g, **f64).mul_(std)

    def oovv_like(std):
        n = o * o * v * v
        out = torch.empty(2 * n, **f64)
        x = normal((o, o, v, v), std)
        ab = out[n:].view(o, o, v, v)
        torch.add(x, x.permute(1, 0, 3, 2), out=ab).mul_(0.5)
        del x
        torch.sub(ab, ab.transpose(2, 3), out=out[:n].view(o, o, v, v))
        return out

    n_o = o * o * v * o
    i_oovo = torch.empty(2 * n_o, **f64)
    ab = i_oovo[n_o:].view(o, o, v, o)
    ab.copy_(normal((o, o, v, o), 5e-2))
    torch.sub(ab, ab.transpose(0, 1), out=i_oovo[:n_o].view(o, o, v, o))

    npr = v * (v - 1) // 2
    n_aa = o * v * npr
    i_ovvv = torch.empty(n_aa + o * v * v * v, **f64)
    abv = i_ovvv[n_aa:].view(o, v, v, v)
    rows, cols = torch.tril_indices(v, v, -1, device=device)
    flat = rows * v + cols
    aav = i_ovvv[:n_aa].view(o, v, npr)
    for k in range(o):   # one k slice at a time keeps temporaries small
        s = abv[k]
        s.copy_(normal((v, v, v), 5e-2))
        d = (s - s.transpose(1, 2)).reshape(v, v * v)
        aav[k].copy_(d.index_select(1, flat))
        del d
    e_i = torch.rand(o, generator=g, **f64) * 1.2 - 1.5
    e_a = torch.rand(v, generator=g, **f64) * 2.9 + 0.1
    tensors = dict(
        d_ov=(e_i[:, None] - e_a[None, :]).reshape(-1).contiguous(),
        f_ov=(normal((o * v,), fock) if fock else torch.zeros(o * v, **f64)),
        t1=normal((o * v,), 1e-3),
        t2=oovv_like(1e-2), i_oovo=i_oovo, i_oovv=oovv_like(5e-2),
        i_ovvv=i_ovvv)
    meta = dict(kind="rpt", oa=o, va=v, ob=o, vb=v)
    return meta, tensors


def restricted_as_unrestricted(case):
    """A restricted case rewritten as the equivalent unrestricted input
    (bbbb = aaaa, baba = abab blocks), whose energy equals the restricted
    one (src/pt.c:469-473 vs 514-529)."""
    o, v = case["oa"], case["va"]
    kind = "upt" if case["kind"] == "rpt" else "uft"
    n4, no, nw = o * o * v * v, o * o * v * o, o * v * v * (v - 1) // 2
    out = dict(kind=kind, oa=o, va=v, ob=o, vb=v)

    def dup_ov(x):
        return np.concatenate([x, x])

    def dup4(x, na):
        aa, ab = x[:na], x[na:]
        return np.concatenate([aa, ab, aa, ab])

    names = (["d_ov", "f_ov", "t1"] if kind == "upt"
             else ["d_ov", "f2_ov", "l1"])
    for n in names:
        out[n] = dup_ov(case[n])
    for n in ("t2", "l2", "i_oovv"):
        if n in case:
            out[n] = dup4(case[n], n4)
    for n in ("i_oovo", "i2_t2f2_oovo", "i6_oovo"):
        if n in case:
            out[n] = dup4(case[n], no)
    for n in ("i_ovvv", "i3_ovvv", "i7_ovvv"):
        if n in case:
            out[n] = dup4(case[n], nw)
    return out


def case_device(kind, oa, va, ob=None, vb=None, seed=0, fock=0.0,
                device="cuda"):
    """Any of the four kinds generated on the GPU with torch (same recipes
    and distributions as the host generators above, not the same numbers),
    for the larger accuracy workloads.  Returns (meta, tensors): pt.h-layout
    float64 CUDA tensors keyed by the pt.h argument names."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    f64 = dict(dtype=torch.float64, device=device)
    restricted = kind[0] == "r"
    if restricted:
        ob, vb = oa, va
    ob = oa if ob is None else ob
    vb = va if vb is None else vb

    def normal(shape, std):
        return torch.randn(shape, generator=g, **f64).mul_(std)

    def energies(o, v):
        ei = torch.rand(o, generator=g, **f64) * 1.2 - 1.5
        ea = torch.rand(v, generator=g, **f64) * 2.9 + 0.1
        return (ei[:, None] - ea[None, :]).reshape(-1)

    def pack(x):
        v = x.shape[-1]
        r, c = torch.tril_indices(v, v, -1, device=device)
        return x.reshape(*x.shape[:-2], v * v).index_select(-1, r * v + c)

    def cat(*blocks):
        return torch.cat([b.reshape(-1) for b in blocks])

    def oovv_like(std):
        if restricted:
            x = normal((oa, oa, va, va), std)
            ab = 0.5 * (x + x.permute(1, 0, 3, 2))
            return cat(ab - ab.transpose(2, 3), ab)
        def same(o, v):
            x = normal((o, o, v, v), std)
            x = x - x.transpose(0, 1)
            return 0.5 * (x - x.transpose(2, 3))
        ab = normal((oa, ob, va, vb), std)
        return cat(same(oa, va), ab, same(ob, vb), ab.permute(1, 0, 3, 2))

    def oovo_like(std):
        if restricted:
            ab = normal((oa, oa, va, oa), std)
            return cat(ab - ab.transpose(0, 1), ab)
        aa = normal((oa, oa, va, oa), std)
        bb = normal((ob, ob, vb, ob), std)
        return cat(aa - aa.transpose(0, 1), normal((oa, ob, va, ob), std),
                   bb - bb.transpose(0, 1), normal((ob, oa, vb, oa), std))

    def ovvv_like(std):
        def same(o, v):   # one occupied slice at a time (temporaries small)
            return torch.cat([pack(s - s.transpose(1, 2))
                              for s in normal((o, v, v, v), std)])
        if restricted:
            ab = normal((oa, va, va, va), std)
            aa = torch.cat([pack(s - s.transpose(1, 2)) for s in ab])
            return cat(aa, ab)
        return cat(same(oa, va), normal((oa, vb, va, vb), std),
                   same(ob, vb), normal((ob, va, vb, va), std))

    nov = oa * va + (0 if restricted else ob * vb)
    d = energies(oa, va) if restricted else torch.cat([energies(oa, va),
                                                       energies(ob, vb)])
    f = normal((nov,), fock) if fock else torch.zeros(nov, **f64)
    meta = dict(kind=kind, oa=oa, va=va, ob=ob, vb=vb)
    if kind[1:] == "pt":
        t = dict(d_ov=d, f_ov=f, t1=normal((nov,), 1e-3),
                 t2=oovv_like(1e-2), i_oovo=oovo_like(5e-2),
                 i_oovv=oovv_like(5e-2), i_ovvv=ovvv_like(5e-2))
    else:
        omega = float(torch.rand(1, generator=g, **f64) * 0.3 + 0.2)
        meta["omega"] = omega
        t = dict(d_ov=d + omega / 3.0, f2_ov=f, l1=normal((nov,), 1e-3),
                 t2=oovv_like(1e-2), l2=oovv_like(1e-2),
                 i_oovv=oovv_like(5e-2), i2_t2f2_oovo=oovo_like(5e-2),
                 i3_ovvv=ovvv_like(5e-2), i6_oovo=oovo_like(5e-2),
                 i7_ovvv=ovvv_like(5e-2))
    return meta, {k: x.contiguous() for k, x in t.items()}
