"""The device producer's conventions (libpt_rpt_inputs_df,
libpt_upt_inputs_df), pinned on the reference's own fixtures, and its numpy
restatements (the checkers of tests/test_gpu_producer.py).

pt.h asks only for "properly (anti-)symmetrized" tensors (src/pt.h:37-57).
The fixtures the reference ships (tests/rpt02.dat, rpt09.dat, converted to
tests/golden/*.npz) come from real molecules; their abab blocks have the
index symmetries of the Mulliken products (ia|jb), (ib|ac), (ia|jk) that a
density-fitted build produces, the oovv one is a positive semidefinite
(ia),(jb) matrix (a Gram matrix of factors), and every aaaa block is its
abab block minus the swapped one -- the relations the producer builds."""
import numpy as np
import pytest

from tests.golden import fixtures


def blocks(case):
    o, v = int(case["oa"]), int(case["va"])
    npr = v * (v - 1) // 2
    n2, n3 = o * o * v * v, o * o * v * o
    return dict(
        o=o, v=v,
        t2_aa=case["t2"][:n2].reshape(o, o, v, v),
        t2_ab=case["t2"][n2:].reshape(o, o, v, v),
        oovv_aa=case["i_oovv"][:n2].reshape(o, o, v, v),
        oovv_ab=case["i_oovv"][n2:].reshape(o, o, v, v),
        oovo_aa=case["i_oovo"][:n3].reshape(o, o, v, o),
        oovo_ab=case["i_oovo"][n3:].reshape(o, o, v, o),
        ovvv_aa=case["i_ovvv"][:o * v * npr].reshape(o, v, npr),
        ovvv_ab=case["i_ovvv"][o * v * npr:].reshape(o, v, v, v))


def df_inputs(b_oo, b_ov, b_vv, t2_abab=None):
    """Numpy restatement of libpt_rpt_inputs_df: the pt.h restricted arrays
    (flat, aaaa block first) from three-index factors."""
    naux, o, v = b_ov.shape
    ab_oovv = np.einsum("qia,qjb->ijab", b_ov, b_ov)
    ab_ovvv = np.einsum("qib,qac->iabc", b_ov, b_vv)
    ab_oovo = np.einsum("qia,qjk->ijak", b_ov, b_oo)
    r, c = np.tril_indices(v, -1)
    out = dict(
        i_oovv=np.concatenate([(ab_oovv - ab_oovv.transpose(0, 1, 3, 2)).ravel(),
                               ab_oovv.ravel()]),
        i_oovo=np.concatenate([(ab_oovo - ab_oovo.transpose(1, 0, 2, 3)).ravel(),
                               ab_oovo.ravel()]),
        i_ovvv=np.concatenate([(ab_ovvv - ab_ovvv.transpose(0, 1, 3, 2))
                               [:, :, r, c].ravel(), ab_ovvv.ravel()]))
    if t2_abab is not None:
        out["t2"] = np.concatenate([
            (t2_abab - t2_abab.transpose(0, 1, 3, 2)).ravel(), t2_abab.ravel()])
    return out


def random_factors(o, v, naux, seed):
    rng = np.random.default_rng(seed)
    b_oo = rng.normal(0, 0.1, (naux, o, o))
    b_oo = 0.5 * (b_oo + b_oo.transpose(0, 2, 1))     # (ij| symmetric in i, j
    b_vv = rng.normal(0, 0.1, (naux, v, v))
    b_vv = 0.5 * (b_vv + b_vv.transpose(0, 2, 1))
    b_ov = rng.normal(0, 0.1, (naux, o, v))
    t2 = rng.normal(0, 1e-2, (o, o, v, v))
    t2 = 0.5 * (t2 + t2.transpose(1, 0, 3, 2))        # t2[ijab] = t2[jiba]
    return b_oo, b_ov, b_vv, t2


@pytest.mark.parametrize("name", ["rpt02", "rpt09"])
def test_reference_fixtures_have_the_produced_structure(name):
    b = blocks(fixtures.load(name))
    tol = 1e-13 * max(np.abs(b["oovv_ab"]).max(), 1.0)
    ab = b["oovv_ab"]
    assert np.abs(ab - ab.transpose(1, 0, 3, 2)).max() <= tol       # (ia|jb)
    gram = ab.transpose(0, 2, 1, 3).reshape(b["o"] * b["v"], -1)
    assert np.linalg.eigvalsh(0.5 * (gram + gram.T)).min() > -1e-12
    ov = b["ovvv_ab"]
    assert np.abs(ov - ov.transpose(0, 3, 2, 1)).max() <= tol       # (ib|ac)
    oo = b["oovo_ab"]
    assert np.abs(oo - oo.transpose(0, 3, 2, 1)).max() <= tol       # (ia|jk)
    assert np.abs(b["oovv_aa"] - (ab - ab.transpose(0, 1, 3, 2))).max() <= tol
    assert np.abs(b["oovo_aa"] - (oo - oo.transpose(1, 0, 2, 3))).max() <= tol
    r, c = np.tril_indices(b["v"], -1)
    assert np.abs(b["ovvv_aa"] -
                  (ov - ov.transpose(0, 1, 3, 2))[:, :, r, c]).max() <= tol
    t2 = b["t2_ab"]
    assert np.abs(b["t2_aa"] - (t2 - t2.transpose(0, 1, 3, 2))).max() <= tol


def test_restatement_builds_that_structure():
    o, v = 3, 7
    b_oo, b_ov, b_vv, t2 = random_factors(o, v, 12, seed=3)
    case = dict(oa=o, va=v, **df_inputs(b_oo, b_ov, b_vv, t2))
    b = blocks(case)
    assert np.allclose(b["oovv_ab"], b["oovv_ab"].transpose(1, 0, 3, 2))
    assert np.allclose(b["ovvv_ab"], b["ovvv_ab"].transpose(0, 3, 2, 1))
    assert np.allclose(b["oovo_ab"], b["oovo_ab"].transpose(0, 3, 2, 1))
    assert np.array_equal(b["t2_ab"], t2)
    # one element of each family by hand
    q = np.arange(12)
    assert np.isclose(b["ovvv_ab"][1, 2, 3, 4],
                      np.sum(b_ov[q, 1, 3] * b_vv[q, 2, 4]))
    assert np.isclose(b["oovo_ab"][0, 2, 5, 1],
                      np.sum(b_ov[q, 0, 5] * b_oo[q, 2, 1]))


def df_inputs_u(fa, fb):
    """Numpy restatement of libpt_upt_inputs_df: the pt.h unrestricted
    integral arrays (blocks aaaa, abab, bbbb, baba) from each spin's factors
    fa, fb = (b_oo, b_ov, b_vv)."""
    def same(oo, ov, vv):
        v = ov.shape[2]
        r, c = np.tril_indices(v, -1)
        g = np.einsum("qia,qjb->ijab", ov, ov)
        y = np.einsum("qia,qjk->ijak", ov, oo)
        z = np.einsum("qib,qac->iabc", ov, vv)
        return ((g - g.transpose(0, 1, 3, 2)).ravel(),
                (y - y.transpose(1, 0, 2, 3)).ravel(),
                (z - z.transpose(0, 1, 3, 2))[:, :, r, c].ravel())

    def mixed(x, y):
        return (np.einsum("qia,qjb->ijab", x[1], y[1]).ravel(),
                np.einsum("qia,qjk->ijak", x[1], y[0]).ravel(),
                np.einsum("qib,qac->iabc", x[1], y[2]).ravel())
    sa, sb, ab, ba = same(*fa), same(*fb), mixed(fa, fb), mixed(fb, fa)
    return dict(i_oovv=np.concatenate([sa[0], ab[0], sb[0], ba[0]]),
                i_oovo=np.concatenate([sa[1], ab[1], sb[1], ba[1]]),
                i_ovvv=np.concatenate([sa[2], ab[2], sb[2], ba[2]]))


def spin_factors(o, v, naux, seed):
    rng = np.random.default_rng(seed)
    oo = rng.normal(0, 0.1, (naux, o, o))
    vv = rng.normal(0, 0.1, (naux, v, v))
    return (0.5 * (oo + oo.transpose(0, 2, 1)), rng.normal(0, 0.1, (naux, o, v)),
            0.5 * (vv + vv.transpose(0, 2, 1)))


@pytest.mark.parametrize("name", ["upt01", "upt03"])
def test_unrestricted_fixtures_have_the_produced_structure(name):
    """abab and baba blocks of the reference's unrestricted fixtures are
    Mulliken products of the same kind: baba oovv is abab's transpose, the
    OVVV mixed blocks are symmetric in their two same-spin virtual indices
    and the OOVO ones in their two same-spin occupied indices."""
    c = fixtures.load(name)
    oa, va, ob, vb = (int(c[k]) for k in ("oa", "va", "ob", "vb"))
    npa, npb = va * (va - 1) // 2, vb * (vb - 1) // 2

    def cut(x, sizes):
        off = np.cumsum([0] + sizes)
        return [x[off[n]:off[n + 1]] for n in range(len(sizes))]
    vv = cut(c["i_oovv"], [oa * oa * va * va, oa * ob * va * vb,
                           ob * ob * vb * vb, ob * oa * vb * va])
    ab, ba = vv[1].reshape(oa, ob, va, vb), vv[3].reshape(ob, oa, vb, va)
    tol = 1e-13 * max(np.abs(ab).max(), 1.0)
    assert np.abs(ba - ab.transpose(1, 0, 3, 2)).max() <= tol
    v3 = cut(c["i_ovvv"], [oa * va * npa, oa * vb * va * vb, ob * vb * npb,
                           ob * va * vb * va])
    for blk, shape in ((v3[1], (oa, vb, va, vb)), (v3[3], (ob, va, vb, va))):
        x = blk.reshape(shape)
        assert np.abs(x - x.transpose(0, 3, 2, 1)).max() <= tol
    vo = cut(c["i_oovo"], [oa * oa * va * oa, oa * ob * va * ob,
                           ob * ob * vb * ob, ob * oa * vb * oa])
    for blk, shape in ((vo[1], (oa, ob, va, ob)), (vo[3], (ob, oa, vb, oa))):
        x = blk.reshape(shape)
        assert np.abs(x - x.transpose(0, 3, 2, 1)).max() <= tol


def test_unrestricted_restatement_with_equal_spins_is_the_restricted_one():
    """With the same factors for both spins, the unrestricted arrays are the
    restricted ones with bbbb = aaaa and baba = abab (the identity the
    restricted path relies on, src/pt.c:469-473)."""
    o, v, q = 3, 6, 9
    f = spin_factors(o, v, q, seed=4)
    u = df_inputs_u(f, f)
    r = df_inputs(*f)
    npr = v * (v - 1) // 2
    assert np.allclose(u["i_oovv"], np.concatenate([r["i_oovv"], r["i_oovv"]]))
    assert np.allclose(u["i_oovo"], np.concatenate([r["i_oovo"], r["i_oovo"]]))
    assert np.allclose(u["i_ovvv"],
                       np.concatenate([r["i_ovvv"][:o * v * npr],
                                       r["i_ovvv"][o * v * npr:],
                                       r["i_ovvv"][:o * v * npr],
                                       r["i_ovvv"][o * v * npr:]]))


def test_producer_entry_points_refuse_bad_arguments_before_any_device_work():
    """Argument checks come first (no pointer is dereferenced, no CUDA call
    made), so they run without a GPU."""
    from libpt_b200 import ffi
    L = ffi.lib()
    p = 4096    # never dereferenced: every call below fails its checks
    assert L.libpt_rpt_inputs_df(0, 2, 2, p, p, p, None, None, p, p, p,
                                 None) == ffi.LIBPT_ERR_ARG
    assert L.libpt_rpt_inputs_df(1, 1, 1, p, p, p, p, None, p, p, p,
                                 None) == ffi.LIBPT_ERR_ARG
    assert L.libpt_rpt_inputs_df(70000, 70000, 1, p, p, p, None, None, p, p,
                                 p, None) == ffi.LIBPT_ERR_ARG
    # unrestricted: a non-empty factor array may not be NULL
    assert L.libpt_upt_inputs_df(2, 3, 1, 4, 5, p, p, p, None, p, p, p, p, p,
                                 None) == ffi.LIBPT_ERR_ARG
    assert L.libpt_upt_inputs_df(2, 3, 0, 4, 5, p, p, p, None, None, None,
                                 p, p, p, None) == ffi.LIBPT_ERR_ARG   # b_vv_b
    assert L.libpt_upt_inputs_df(2, 3, 1, 4, 0, p, p, p, p, p, p, p, p, p,
                                 None) == ffi.LIBPT_ERR_ARG             # naux 0
    assert b"libpt_upt_inputs_df" in L.libpt_last_error()
