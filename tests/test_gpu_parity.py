"""GPU parity: the device library against the reference's golden vectors and
against the oracle (the reference build oracle/_ref when present, else our C
restatement) on the same seeded inputs.

Tolerances:
  golden fixtures, FP64 and FP32 entry points: |dE| <= 1e-8 Eh (test.cpp:29)
  FP64 vs the reference's own FP64 value:      |dE| <= 1e-9 Eh and
                                               |dE| <= 1e-12 |E|
  FP32 (*_mp) entry points (the FP32 tensor-core form): at the FP32-input
  floor, |dE| <= 1.25 max(|Emp - E64|, |E64(fl x) - E64|) against the
  reference FP64 energy, with the reference's own *_mp error and the
  rounding of the FP32 inputs (fl x) as the two yardsticks; the form's
  arithmetic error alone is bounded in tests/test_gpu_fp32.py
"""
import os

import numpy as np
import pytest

from libpt_b200 import ffi, synth
from oracle import oracle
from tests.golden import fixtures

pytestmark = pytest.mark.gpu

GOLDEN_EPS = 1e-8
ABS64, REL64 = 1e-9, 1e-12


def checker():
    if os.path.exists(oracle.reference_path()):
        return oracle.reference()
    return oracle.restatement()


@pytest.fixture(scope="module")
def energies():
    return fixtures.energies()


def close64(e, ref):
    return abs(e - ref) <= ABS64 and abs(e - ref) <= REL64 * abs(ref) + 1e-15


def to_dev(case, mp=False):
    import torch
    dt = torch.float32 if mp else torch.float64
    return {n: torch.as_tensor(np.ascontiguousarray(case[n])).to(
        device="cuda", dtype=dt) for n in ffi.args_of(case["kind"])}


@pytest.mark.parametrize("name", fixtures.NAMES)
def test_golden_fp64(name, energies):
    case = fixtures.load(name)
    e = ffi.solve_host(case)
    assert abs(e - case["e_ref"]) <= GOLDEN_EPS
    assert close64(e, energies[name]["ref_fp64"])


def rounded(case):
    """The case's inputs rounded to FP32 (as FP64 arrays)."""
    out = dict(case)
    for k in oracle.args_of(case["kind"]):
        out[k] = np.asarray(case[k], np.float32).astype(np.float64)
    return out


def mp_floor_bar(e, e64, emp, e64_in):
    """|e - E64| within the FP32-input floor: the reference *_mp's own
    error or the input rounding, whichever is larger (x 1.25)."""
    return abs(e - e64) <= 1.25 * max(abs(emp - e64), abs(e64_in - e64)) \
        + 1e-16


@pytest.mark.parametrize("name", fixtures.NAMES)
def test_golden_mp(name, energies):
    case = fixtures.load(name)
    e = ffi.solve_host(case, mp=True)
    assert abs(e - case["e_ref"]) <= GOLDEN_EPS
    e64_in = oracle.solve(checker(), rounded(case))
    ref = energies[name]
    assert mp_floor_bar(e, ref["ref_fp64"], ref["ref_fp32"], e64_in), \
        (e - ref["ref_fp64"], ref["ref_fp32"] - ref["ref_fp64"],
         e64_in - ref["ref_fp64"])


SYNTH = [
    ("rpt", (5, 13)), ("rpt", (6, 20)), ("rpt", (8, 64)), ("rpt", (3, 2)),
    ("rpt", (1, 6)), ("rpt", (2, 7)), ("rpt", (7, 33)), ("rpt", (4, 130)),
    ("rpt", (20, 17)),
    ("upt", (4, 11, 3, 13)), ("upt", (2, 3, 5, 8)), ("upt", (1, 5, 2, 6)),
    ("upt", (6, 29, 5, 31)),
    ("rft", (4, 10)), ("rft", (6, 37)),
    ("uft", (3, 9, 4, 7)), ("uft", (2, 5, 1, 4)), ("uft", (5, 21, 4, 18)),
]


@pytest.mark.parametrize("kind,sz", SYNTH)
def test_synthetic_fp64_vs_oracle(kind, sz):
    case = synth.make(kind, *sz, seed=21, fock=1e-3)
    ref = oracle.solve(checker(), case)
    e = ffi.solve_host(case)
    assert close64(e, ref), (e, ref, e - ref)


@pytest.mark.parametrize("kind,sz", [("rpt", (5, 13)), ("upt", (4, 11, 3, 13)),
                                     ("rft", (4, 10)), ("uft", (3, 9, 4, 7))])
def test_synthetic_mp_vs_oracle(kind, sz):
    case = synth.make(kind, *sz, seed=22, fock=1e-3)
    e64 = oracle.solve(checker(), case)
    emp = oracle.solve(checker(), case, mp=True)
    e64_in = oracle.solve(checker(), rounded(case))
    e = ffi.solve_host(case, mp=True)
    assert mp_floor_bar(e, e64, emp, e64_in), (e - e64, emp - e64,
                                               e64_in - e64)


@pytest.mark.parametrize("kind,sz", [("rpt", (5, 13)), ("upt", (4, 11, 3, 13)),
                                     ("rft", (4, 10)), ("uft", (3, 9, 4, 7))])
def test_device_twin_equals_host_entry(kind, sz):
    case = synth.make(kind, *sz, seed=23, fock=1e-3)
    e_host = ffi.solve_host(case)
    e_dev = ffi.solve_device(case, to_dev(case))
    assert e_dev == e_host          # same engine, same order: bitwise
    e_mp = ffi.solve_device(case, to_dev(case, mp=True), mp=True)
    assert e_mp == ffi.solve_host(case, mp=True)


@pytest.mark.parametrize("kind,sz,fock", [
    ("rpt", (2, 9), 0.0), ("rpt", (3, 17), 1e-3), ("rpt", (7, 33), 0.0),
    ("rft", (2, 8), 1e-3), ("rft", (5, 21), 0.0)])
def test_streamed_host_upload_equals_device_inputs(kind, sz, fock):
    """Restricted FP64 host-array solves copy i_ovvv (and i3/i7_ovvv) by
    occupied index beside the triples that need them: the energy is the
    device-input energy bitwise, including queues whose first indices own
    no triple (o = 2, 3) and a nonzero f_ov."""
    case = synth.make(kind, *sz, seed=31, fock=fock)
    assert ffi.solve_host(case) == ffi.solve_device(case, to_dev(case))


def test_zero_sizes():
    for kind, sz in [("rpt", (0, 5)), ("rpt", (3, 0)), ("rpt", (3, 1)),
                     ("upt", (2, 3, 0, 4)), ("uft", (0, 3, 2, 4))]:
        case = synth.make(kind, *sz, seed=1)
        assert ffi.solve_host(case) == oracle.solve(oracle.restatement(), case)


def test_plan_pieces_equal_whole_and_are_deterministic():
    case = synth.make("upt", 5, 17, 4, 19, seed=5, fock=1e-3)
    t = to_dev(case)
    p = ffi.Plan(case, t)
    p.run()
    e_all = p.energy()
    q = ffi.Plan(case, t)
    order = np.random.default_rng(0).permutation(q.n)
    for chunk in np.array_split(order, 7):
        q.run(chunk)
    assert q.energy() == e_all
    assert close64(e_all, oracle.solve(checker(), case))
    # subset energies: sum over disjoint halves equals the whole
    half = np.arange(q.n // 2)
    rest = np.arange(q.n // 2, q.n)
    assert q.energy(half) + q.energy(rest) == pytest.approx(e_all, rel=1e-14)
    p.close()
    q.close()


def test_per_triple_energies_match_oracle():
    case = synth.rpt_case(6, 21, seed=9, fock=1e-3)
    p = ffi.Plan(case, to_dev(case))
    p.run()
    ref = np.concatenate([oracle.rpt_partials(case, 0),
                          oracle.rpt_partials(case, 1)])
    assert p.n == ref.size
    got = np.array([p.energy([q]) for q in range(p.n)]) / 2.0
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-16)


def test_repeat_is_bitwise_identical():
    case = synth.make("rft", 5, 23, seed=31, fock=1e-3)
    assert ffi.solve_host(case) == ffi.solve_host(case)


@pytest.mark.parametrize("name", fixtures.NAMES)
def test_golden_tf32x3_plan(name, energies):
    """The 3xTF32 tensor-core form on the golden fixtures (FP32 inputs)."""
    case = fixtures.load(name)
    p = ffi.Plan(case, to_dev(case, mp=True), mp=True,
                 precision=ffi.PREC_TF32X3)
    p.run()
    e = p.energy()
    p.close()
    assert abs(e - case["e_ref"]) <= GOLDEN_EPS


@pytest.mark.parametrize("kind,sz", [("rpt", (6, 40)), ("upt", (4, 23, 3, 25)),
                                     ("rft", (4, 21)), ("uft", (3, 17, 4, 19))])
def test_synthetic_tf32x3_plan(kind, sz):
    """Stated tolerance of the 3xTF32 form: |dE| <= 2e-5 |E|."""
    case = synth.make(kind, *sz, seed=24, fock=1e-3)
    ref = oracle.solve(checker(), case)
    p = ffi.Plan(case, to_dev(case, mp=True), mp=True,
                 precision=ffi.PREC_TF32X3)
    p.run()
    e = p.energy()
    p.close()
    assert abs(e - ref) <= 2e-5 * abs(ref)


@pytest.mark.parametrize("name", fixtures.NAMES)
def test_golden_emulated_fp64(name, energies):
    """Emulated FP64 (6 slices) on the golden fixtures: the reference FP64
    value to 1e-12 Eh (measured <= 1e-14)."""
    case = fixtures.load(name)
    p = ffi.Plan(case, to_dev(case), precision=ffi.PREC_EMU64 | (6 << 8))
    p.run()
    e = p.energy()
    p.close()
    assert abs(e - energies[name]["ref_fp64"]) <= 1e-12


@pytest.mark.parametrize("kind,sz", [("rpt", (8, 64)), ("upt", (5, 21, 4, 23)),
                                     ("rft", (5, 30)), ("uft", (4, 17, 3, 19))])
def test_synthetic_emulated_fp64(kind, sz):
    """Stated tolerance of emulated FP64 (6 slices): |dE| <= 1e-6 Eh against
    the reference FP64, and <= 1e-11 |E| + 1e-13 Eh (measured <= 9e-12 Eh on
    |E| ~ 1e1, 3e-14 Eh on |E| ~ 5e-3)."""
    case = synth.make(kind, *sz, seed=5, fock=1e-3)
    ref = oracle.solve(checker(), case)
    p = ffi.Plan(case, to_dev(case), precision=ffi.PREC_EMU64 | (6 << 8))
    p.run()
    e = p.energy()
    p.close()
    assert abs(e - ref) <= 1e-6
    assert abs(e - ref) <= 1e-11 * abs(ref) + 1e-13


@pytest.mark.parametrize("kind,sz", [("rpt", (8, 64)), ("upt", (5, 21, 4, 23)),
                                     ("rft", (5, 30)), ("uft", (4, 17, 3, 19)),
                                     ("rpt", (12, 90))])
def test_emulated_fp64_chosen_slices_meet_1_uEh(kind, sz):
    """Slice count left to the plan (S = 0): the chosen S keeps |dE| within
    the 1 uEh target against the reference FP64 value."""
    case = synth.make(kind, *sz, seed=6, fock=1e-3)
    ref = oracle.solve(checker(), case)
    p = ffi.Plan(case, to_dev(case), precision=ffi.PREC_EMU64)
    p.run()
    e = p.energy()
    p.close()
    assert abs(e - ref) <= 1e-6, (e, ref)


@pytest.mark.parametrize("kind,sz", [("rpt", (20, 60)), ("upt", (14, 50, 12, 52)),
                                     ("rft", (16, 40)), ("uft", (12, 30, 11, 33))])
def test_emulated_fp64_sampled_slice_choice_meets_1_uEh(kind, sz):
    """Queues long enough for the sampled choice (N >= 640 triples): the S
    the error estimate picks keeps |dE| <= 1 uEh against the FP64 path
    (which matches the reference to 1e-12 |E|), and the worst-case bound
    never picks fewer slices than the estimate."""
    import os
    import subprocess
    import sys
    case = synth.make(kind, *sz, seed=8, fock=1e-3)
    dev = to_dev(case)
    p64 = ffi.Plan(case, dev)
    p64.run()
    e64 = p64.energy()
    p64.close()
    p = ffi.Plan(case, dev, precision=ffi.PREC_EMU64)
    assert p.n >= 640
    p.run()
    e, s_est = p.energy(), p.slices
    p.close()
    assert 4 <= s_est <= 7
    assert abs(e - e64) <= 1e-6, (s_est, e, e64)
    code = (f"import sys; sys.path.insert(0, {os.getcwd()!r})\n"
            "from libpt_b200 import ffi, synth\n"
            "from tests.test_gpu_parity import to_dev\n"
            f"case = synth.make({kind!r}, *{sz!r}, seed=8, fock=1e-3)\n"
            "p = ffi.Plan(case, to_dev(case), precision=ffi.PREC_EMU64)\n"
            "print(p.slices)\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True,
                       text=True, timeout=600,
                       env=dict(os.environ, LIBPT_EMU_BOUND="worst"))
    assert r.returncode == 0, r.stderr
    assert int(r.stdout.strip().splitlines()[-1]) >= s_est


@pytest.mark.parametrize("digits", [7, 8])
def test_emulated_fp64_digit_prefix_equals_fixed_slices(digits):
    """A plan that chose S runs on the first S of its stored digit planes.
    With 7-bit digits they are exactly the S-slice decomposition: the energy
    equals that of a plan built with S slices, bitwise.  With 8-bit digits
    they differ from it only where a carry from a lower digit changed the
    last kept digit, within the same error bound."""
    import os
    # 1012 triples: long enough for the sampled choice
    case = synth.make("rpt", 12, 30, seed=8, fock=1e-3)
    os.environ["LIBPT_EMU_TOL"] = "1e3"          # loose: the choice is S = 4
    os.environ["LIBPT_EMU_DIGITS"] = str(digits)
    try:
        p = ffi.Plan(case, to_dev(case), precision=ffi.PREC_EMU64)
        assert p.slices == 4
        p.run()
        e_auto = p.energy()
        p.close()
        q = ffi.Plan(case, to_dev(case), precision=ffi.PREC_EMU64 | (4 << 8))
        q.run()
        e4 = q.energy()
        q.close()
    finally:
        del os.environ["LIBPT_EMU_TOL"]
        del os.environ["LIBPT_EMU_DIGITS"]
    if digits == 7:
        assert e_auto == e4
    else:
        assert abs(e_auto - e4) <= 1e-9 * abs(e4), (e_auto, e4)
