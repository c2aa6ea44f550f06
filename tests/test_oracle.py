"""CPU tests: the oracle is pinned to the reference's golden vectors and to the
reference library itself (oracle/_ref, compiled from its own sources)."""
import os

import numpy as np
import pytest

from libpt_b200 import synth
from oracle import oracle
from tests.golden import fixtures

GOLDEN_EPS = 1e-8   # test.cpp:29


def have_ref():
    return os.path.exists(oracle.reference_path())


@pytest.fixture(scope="module")
def energies():
    return fixtures.energies()


@pytest.mark.parametrize("name", fixtures.NAMES)
@pytest.mark.parametrize("mp", [False, True])
def test_restatement_matches_golden_header(name, mp, energies):
    """Same check as the reference's `make check` (test.cpp:988-991)."""
    case = fixtures.load(name)
    e = oracle.solve(oracle.restatement(), case, mp=mp)
    assert abs(e - case["e_ref"]) <= GOLDEN_EPS


@pytest.mark.parametrize("name", fixtures.NAMES)
def test_restatement_matches_reference_full_precision(name, energies):
    """FP64 restatement vs the reference library's own value, to rounding."""
    case = fixtures.load(name)
    e = oracle.solve(oracle.restatement(), case)
    ref = energies[name]["ref_fp64"]
    assert abs(e - ref) <= 1e-14 * abs(ref) + 1e-18
    e32 = oracle.solve(oracle.restatement(), case, mp=True)
    assert abs(e32 - energies[name]["ref_fp32"]) <= 1e-5 * abs(ref) + 1e-12


@pytest.mark.skipif(not have_ref(), reason="reference build absent")
@pytest.mark.parametrize("name", fixtures.NAMES)
def test_reference_build_reproduces_golden(name, energies):
    case = fixtures.load(name)
    for mp in (False, True):
        e = oracle.solve(oracle.reference(), case, mp=mp)
        assert abs(e - case["e_ref"]) <= GOLDEN_EPS
    assert oracle.solve(oracle.reference(), case) == pytest.approx(
        energies[name]["ref_fp64"], rel=1e-13, abs=1e-18)


SYNTH = [
    ("rpt", (5, 13)), ("rpt", (4, 9)), ("rpt", (3, 2)), ("rpt", (1, 6)),
    ("upt", (4, 11, 3, 13)), ("upt", (2, 3, 5, 8)), ("upt", (1, 5, 2, 6)),
    ("rft", (4, 10)), ("uft", (3, 9, 4, 7)), ("uft", (2, 5, 1, 4)),
]


@pytest.mark.skipif(not have_ref(), reason="reference build absent")
@pytest.mark.parametrize("kind,sz", SYNTH)
def test_restatement_matches_reference_synthetic(kind, sz):
    case = synth.make(kind, *sz, seed=11, fock=1e-3)
    e_ref = oracle.solve(oracle.reference(), case)
    e = oracle.solve(oracle.restatement(), case)
    assert abs(e - e_ref) <= 1e-13 * abs(e_ref) + 1e-18
    f_ref = oracle.solve(oracle.reference(), case, mp=True)
    f = oracle.solve(oracle.restatement(), case, mp=True)
    assert abs(f - f_ref) <= 1e-5 * abs(e_ref) + 1e-12


@pytest.mark.parametrize("kind", ["rpt", "rft"])
def test_restricted_equals_closed_shell_unrestricted(kind):
    """rpt = upt and rft = uft when beta blocks equal alpha blocks
    (src/pt.c:469-473 vs 514-529; 958-966 vs 1023-1044)."""
    case = synth.make(kind, 5, 11, seed=3, fock=1e-3)
    u = synth.restricted_as_unrestricted(case)
    O = oracle.restatement()
    assert oracle.solve(O, case) == pytest.approx(oracle.solve(O, u),
                                                  rel=1e-13)


def test_empty_spaces_give_zero():
    """src/pt.c:195-196, 318-319: empty spaces contribute nothing."""
    O = oracle.restatement()
    assert oracle.solve(O, synth.make("rpt", 3, 1, seed=1)) == 0.0
    assert oracle.solve(O, synth.make("upt", 2, 3, 0, 4, seed=1)) == 0.0


def test_partials_sum_to_energy():
    case = synth.rpt_case(5, 9, seed=4, fock=1e-3)
    p0 = oracle.rpt_partials(case, 0)
    p1 = oracle.rpt_partials(case, 1)
    assert len(p0) == 10 and len(p1) == 50
    e = oracle.solve(oracle.restatement(), case)
    assert 2.0 * (p0.sum() + p1.sum()) == pytest.approx(e, rel=1e-13)


def test_synthetic_symmetries():
    o, v = 4, 7
    c = synth.rpt_case(o, v, seed=5)
    n = o * o * v * v
    t2aa = c["t2"][:n].reshape(o, o, v, v)
    t2ab = c["t2"][n:].reshape(o, o, v, v)
    np.testing.assert_allclose(t2ab, t2ab.transpose(1, 0, 3, 2), atol=0)
    np.testing.assert_allclose(t2aa, -t2aa.transpose(0, 1, 3, 2), atol=0)
    np.testing.assert_allclose(t2aa, -t2aa.transpose(1, 0, 2, 3), atol=1e-18)
    np.testing.assert_allclose(t2aa, t2ab - t2ab.transpose(0, 1, 3, 2))
    d = c["d_ov"].reshape(o, v)
    assert (d < 0).all()
    u = synth.upt_case(3, 5, 2, 6, seed=5)
    sizes = [3 * 3 * 5 * 5, 3 * 2 * 5 * 6, 2 * 2 * 6 * 6, 2 * 3 * 6 * 5]
    b = np.split(u["t2"], np.cumsum(sizes)[:-1])
    ab = b[1].reshape(3, 2, 5, 6)
    ba = b[3].reshape(2, 3, 6, 5)
    np.testing.assert_array_equal(ba, ab.transpose(1, 0, 3, 2))
    aa = b[0].reshape(3, 3, 5, 5)
    np.testing.assert_allclose(aa, -aa.transpose(1, 0, 2, 3), atol=1e-18)
