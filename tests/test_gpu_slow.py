"""Full solves at the precision-table sizes (minutes of GPU time each; run
with LIBPT_SLOW_TESTS=1).

* Unrestricted (T) oa=20 va=180 ob=18 vb=182 and unrestricted (fT) o=15
  v=150 per spin against the reference build's energies of the same
  host-generated inputs (tests/golden/reference_energies.json, written by
  tests/golden/make_reference_energies.py with the input SHA-256): FP64 to
  1e-12 |E|, emulated FP64 with the slice count chosen for 1 uEh to 1 uEh,
  and the FP32 tensor-core form on the FP32-rounded inputs with its
  arithmetic error below a tenth of the reference *_mp's.
* Restricted (fT) o=30 v=300, which the reference would need hours for:
  its FP64 energy equals that of the same input written as an unrestricted
  closed-shell case (src/pt.c:958-966 vs 1023-1044), to 1e-12 |E|.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from libpt_b200 import ffi, synth

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

HERE = os.path.dirname(os.path.abspath(__file__))
REL64 = 1e-12


def reference_energies():
    with open(os.path.join(HERE, "golden", "reference_energies.json")) as fp:
        return json.load(fp)


def digest(case):
    h = hashlib.sha256()
    for n in ffi.args_of(case["kind"]):
        h.update(np.ascontiguousarray(case[n], dtype=np.float64).tobytes())
    return h.hexdigest()


def plan_energy(case, tensors, mp=False, precision=ffi.PREC_FP64):
    p = ffi.Plan(case, tensors, mp=mp, precision=precision)
    try:
        p.run()
        return p.energy()
    finally:
        p.close()


@pytest.mark.parametrize("name,kind,sz", [
    ("upt_20_180_18_182", "upt", (20, 180, 18, 182)),
    ("uft_15_150", "uft", (15, 150, 15, 150))])
def test_precision_case_against_reference(name, kind, sz):
    import torch
    ref = reference_energies()[name]
    case = synth.make(kind, *sz, seed=ref["seed"])
    assert digest(case) == ref["input_sha256"]
    dev = {n: torch.as_tensor(np.ascontiguousarray(case[n])).to(
        device="cuda", dtype=torch.float64) for n in ffi.args_of(kind)}
    e_ref, e_mp = ref["fp64"]["energy"], ref["fp32_mp"]["energy"]
    e64 = plan_energy(case, dev)
    assert abs(e64 - e_ref) <= REL64 * abs(e_ref), (e64, e_ref)
    e_emu = plan_energy(case, dev, precision=ffi.PREC_EMU64)
    assert abs(e_emu - e_ref) <= 1e-6, (e_emu, e_ref)
    dev32 = {k: x.float() for k, x in dev.items()}
    del dev
    e_floor = plan_energy(case, dev32, mp=True)
    e_tc = plan_energy(case, dev32, mp=True, precision=ffi.PREC_FP32)
    assert abs(e_tc - e_floor) <= abs(e_mp - e_floor) / 10, \
        (e_tc - e_floor, e_mp - e_floor)
    assert abs(e_tc - e_ref) <= 1.25 * max(abs(e_mp - e_ref),
                                           abs(e_floor - e_ref))


def test_rft_30_300_equals_uft_closed_shell():
    import torch
    meta, t = synth.case_device("rft", 30, 300, seed=11)
    e_r = plan_energy(meta, t)
    o, v = 30, 300
    n4, no, nw = o * o * v * v, o * o * v * o, o * v * v * (v - 1) // 2

    def dup(x, na):   # [aaaa, abab] -> [aaaa, abab, bbbb = aaaa, baba = abab]
        return torch.cat([x, x[:na], x[na:]])

    u = {}
    for n, x in t.items():
        if n in ("d_ov", "f2_ov", "l1"):
            u[n] = torch.cat([x, x])
        elif n in ("t2", "l2", "i_oovv"):
            u[n] = dup(x, n4)
        elif n in ("i2_t2f2_oovo", "i6_oovo"):
            u[n] = dup(x, no)
        else:
            u[n] = dup(x, nw)
    del t
    torch.cuda.empty_cache()
    e_u = plan_energy(dict(kind="uft", oa=o, va=v, ob=o, vb=v), u)
    assert abs(e_u - e_r) <= REL64 * abs(e_r), (e_u, e_r)
