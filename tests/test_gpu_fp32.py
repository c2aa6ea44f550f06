"""The FP32 tensor-core form (LIBPT_PREC_FP32, the default of the *_mp entry
points) against the reference's own FP32 path (src/ptmp.c, built from its
sources as oracle/_ref).

The FP32 entry points receive FP32 inputs, so every FP32 method carries
the rounding of its inputs: d_in = E64(fl x) - E64(x), with E64 the
reference's FP64 solver and fl x the inputs rounded to FP32.  The
reference's *_mp adds its FP32 arithmetic error d_ref = Emp(fl x) -
E64(fl x); the FP32 form adds d_tc = Etc(fl x) - E64(fl x).  Bars:

  arithmetic   |d_tc| <= |d_ref| / 10  (5 INT8 digit planes carry 39 bits,
               digits rounded to nearest: unbiased and far below FP32
               rounding; measured |d_tc / d_ref| <= 0.0075 over these cases,
               where 4 planes reached 0.73 on small systems)
  end to end   |Etc - E64(x)| <= 1.25 max(|Emp - E64(x)|, |d_in|), i.e. at
               the FP32-input floor, within the reference *_mp's own error
               or the input rounding, whichever is larger (the input
               rounding alone exceeds the reference *_mp's total error on
               some of these cases: its arithmetic error partly cancels it)

The 3xTF32 form (opt-in) keeps its own bar: its truncating FP32
accumulation leaves ~2e-6 |E|.
"""
import os

import numpy as np
import pytest

from libpt_b200 import ffi, synth
from oracle import oracle

pytestmark = pytest.mark.gpu

CASES = [("rpt", (5, 13), 22), ("upt", (4, 11, 3, 13), 22),
         ("rft", (4, 10), 22), ("uft", (3, 9, 4, 7), 22),
         ("rpt", (8, 64), 7), ("rpt", (8, 64), 22), ("rpt", (10, 48), 22),
         ("upt", (6, 29, 5, 31), 22), ("rft", (6, 37), 22),
         ("uft", (5, 21, 4, 18), 22)]


def reference():
    if not os.path.exists(oracle.reference_path()):
        pytest.skip("oracle/_ref (the reference build) is not present")
    return oracle.reference()


def rounded(case):
    out = dict(case)
    for k in oracle.args_of(case["kind"]):
        out[k] = np.asarray(case[k], np.float32).astype(np.float64)
    return out


def to_dev(case, mp):
    import torch
    dt = torch.float32 if mp else torch.float64
    return {n: torch.as_tensor(np.ascontiguousarray(case[n])).to(
        device="cuda", dtype=dt) for n in ffi.args_of(case["kind"])}


@pytest.mark.parametrize("kind,sz,seed", CASES)
def test_fp32_form_against_reference_mp(kind, sz, seed):
    ref = reference()
    case = synth.make(kind, *sz, seed=seed, fock=1e-3 if seed == 22 else 0.0)
    e64 = oracle.solve(ref, case)
    e64_in = oracle.solve(ref, rounded(case))
    emp = oracle.solve(ref, case, mp=True)
    etc = ffi.solve_host(case, mp=True)      # default: the FP32 form
    d_in, d_ref, d_tc = e64_in - e64, emp - e64_in, etc - e64_in
    assert abs(d_tc) <= abs(d_ref) / 10, (d_tc, d_ref)
    assert abs(etc - e64) <= 1.25 * max(abs(emp - e64), abs(d_in)), \
        (etc - e64, emp - e64, d_in)


@pytest.mark.parametrize("kind,sz,seed", CASES[:4])
def test_fp32_form_device_twin_and_plan(kind, sz, seed):
    """The _mp device twin and a plan created with LIBPT_PREC_FP32 give the
    host entry point's energy bitwise, and the plan reports 5 slices."""
    case = synth.make(kind, *sz, seed=seed, fock=1e-3)
    e_host = ffi.solve_host(case, mp=True)
    dev = to_dev(case, mp=True)
    assert ffi.solve_device(case, dev, mp=True) == e_host
    p = ffi.Plan(case, dev, mp=True, precision=ffi.PREC_FP32)
    try:
        assert p.slices == 5
        p.run()
        assert p.energy() == e_host
    finally:
        p.close()


def test_fp32_form_rejects_other_slice_counts():
    case = synth.make("rpt", 3, 7, seed=1)
    with pytest.raises(ffi.LibptError):
        ffi.Plan(case, to_dev(case, mp=True), mp=True,
                 precision=ffi.PREC_FP32 | (4 << 8))


def test_mp_precision_override_runs_fp64_engine():
    """LIBPT_MP_PRECISION=fp64 evaluates the FP32 inputs with the FP64
    engine: the reference FP64 energy of the FP32-rounded inputs."""
    import subprocess
    import sys
    ref = reference()
    case = synth.make("rpt", 5, 13, seed=22, fock=1e-3)
    e64_in = oracle.solve(ref, rounded(case))
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from libpt_b200 import ffi, synth\n"
            "case = synth.make('rpt', 5, 13, seed=22, fock=1e-3)\n"
            "print(repr(ffi.solve_host(case, mp=True)))\n" % os.getcwd())
    r = subprocess.run([sys.executable, "-c", code], capture_output=True,
                       text=True, timeout=300,
                       env=dict(os.environ, LIBPT_MP_PRECISION="fp64"))
    assert r.returncode == 0, r.stderr
    e = float(r.stdout.strip().splitlines()[-1])
    assert abs(e - e64_in) <= 1e-12 * abs(e64_in)
