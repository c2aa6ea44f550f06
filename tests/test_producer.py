"""The device producer's conventions (libpt_rpt_inputs_df), pinned on the
reference's own restricted fixtures, and its numpy restatement (the checker
of tests/test_gpu_producer.py).

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
