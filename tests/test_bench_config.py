"""bench.py's workload description: both arms print the same config, and its
flops are the reference's dgemm_ flops of the sampled triples (with stride 1,
the whole queue: rpt_flops(o, v), src/pt.c:49-158).  Also the CPU baseline's
full-solve extrapolation and the accuracy report's fixed-order reference run."""
import sys

import bench


def args_of(*argv):
    old = sys.argv
    sys.argv = ["bench.py", *argv]
    try:
        return bench.parse()
    finally:
        sys.argv = old


def test_default_workload_is_the_o45_v477_sample():
    c = bench.workload_config(args_of(), 1)
    assert c["workload"].startswith("rpt o=45 v=477: every 211th triple of the "
                                    "58740-entry queue")
    assert "(279 triples, 68 same-spin)" in c["workload"]
    assert c["parallelism"] == "1 GPU"


def test_stride_one_covers_the_queue_flops():
    for o, v in ((2, 477), (5, 13), (45, 477)):
        a = args_of("--o", str(o), "--v", str(v), "--stride", "1")
        c = bench.workload_config(a, 1)
        assert abs(c["flops_per_step"] - bench.rpt_flops(o, v)) <= \
            1e-12 * bench.rpt_flops(o, v)


def test_sharded_sample_is_denser_with_ranks():
    one = bench.workload_config(args_of(), 1)
    eight = bench.workload_config(args_of(), 8)
    assert "every 26th" in eight["workload"]
    assert eight["flops_per_step"] > 7 * one["flops_per_step"]
    assert eight["parallelism"].startswith("triples sharded x8")


def test_cpu_extrapolation_scales_each_kind_by_its_rate():
    """Same-spin triples at the same-spin rate, mixed-spin triples at the
    mixed-spin rate: with equal rates the extrapolation is the workload's
    flops over that rate; the triple counts are C(o,3) and C(o,2) o."""
    a = args_of()
    v = 477
    r = dict(flops_aaa=bench.aaa_flops(3, v), seconds_aaa=bench.aaa_flops(3, v) / 0.08e12,
             flops_aab=bench.aab_flops(2, v, 1, v),
             seconds_aab=bench.aab_flops(2, v, 1, v) / 0.08e12)
    x = bench.extrapolation(a, r)
    assert abs(x["extrapolated_solve_seconds"] -
               bench.rpt_flops(45, 477) / 0.08e12) < 1e-6 * x["extrapolated_solve_seconds"]
    assert x["extrapolation"].startswith("extrapolated: rpt o=45 v=477")
    # a mixed-spin rate twice as high halves the mixed-spin part
    r2 = dict(r, seconds_aab=r["seconds_aab"] / 2)
    t_aaa = 14190 * bench.aaa_flops(45, v) / 0.08e12
    t_aab = 44550 * bench.aab_flops(45, v, 45, v) / 0.08e12
    assert abs(bench.extrapolation(a, r2)["extrapolated_solve_seconds"] -
               (t_aaa + t_aab / 2)) < 1e-6 * t_aaa
    assert abs(14190 * bench.aaa_flops(45, v) + 44550 * bench.aab_flops(45, v, 45, v)
               - bench.rpt_flops(45, v)) < 1e-9 * bench.rpt_flops(45, v)


def test_reference_single_thread_run_matches_the_threaded_one():
    """The accuracy report's fixed-order reference (one OpenMP and one BLAS
    thread) and the OpenMP-over-triples run agree to summation-order noise."""
    import os

    import pytest
    from oracle import oracle
    if not os.path.exists(oracle.reference_path()):
        pytest.skip("reference build absent")
    r1 = bench.run_cpu(3, 24, 1, "single")
    rn = bench.run_cpu(3, 24, 1, "omp")
    assert r1["cores"] == 1 and r1["threads"] == "single"
    assert r1["energy"] != 0.0
    assert abs(r1["energy"] - rn["energy"]) <= 1e-12 * abs(r1["energy"])


def test_precision_forms_cover_every_form():
    from libpt_b200 import ffi
    forms = bench.precision_forms(ffi, (4, 5, 6, 7))
    names = [f[0] for f in forms]
    assert names == ["fp64", "emu64_s4", "emu64_s5", "emu64_s6", "emu64_s7",
                     "emu64_auto", "fp32_tc", "fp64_on_fp32_inputs", "tf32x3"]
    # the FP32-input forms: the FP32 tensor-core form, its floor, 3xTF32
    assert [f[0] for f in forms if f[2]] == ["fp32_tc", "fp64_on_fp32_inputs",
                                             "tf32x3"]
    assert dict((f[0], f[1]) for f in forms)["fp32_tc"] == ffi.PREC_FP32


def test_precision_cases_have_reference_energies():
    """Every case of the precision table has committed reference energies
    (FP64 and the reference's FP32 *_mp) for the seed the bench uses."""
    refs = bench.reference_energies()
    for name, kind, sz, seed in bench.PRECISION_CASES:
        if name not in refs:
            import pytest
            pytest.skip(f"{name}: reference energies not generated yet")
        r = refs[name]
        assert r["kind"] == kind and tuple(r["sizes"]) == sz
        assert r["seed"] == seed
        assert r["fp64"]["energy"] != 0.0 and r["fp32_mp"]["energy"] != 0.0


def test_served_inputs_are_windows_of_the_pt_h_sizes():
    """Every request of the served stream gets arrays of the pt.h lengths
    (those of synth.rpt_case), its large ones inside the shared pools, and
    two requests of one size get different windows."""
    import numpy as np
    import torch
    from libpt_b200 import synth
    reqs = [dict(o=3, v=20, seed=1), dict(o=3, v=20, seed=2),
            dict(o=4, v=31, seed=3)]
    cases, pool_gb, own_gb = bench.serve_inputs(reqs, torch)
    for r, c in zip(reqs, cases):
        ref = synth.rpt_case(r["o"], r["v"], seed=0)
        for k, n in bench.rpt_lengths(r["o"], r["v"]).items():
            assert c[k].size == ref[k].size == n, k
            assert c[k].dtype == np.float64 and c[k].flags.c_contiguous
        assert (c["d_ov"] < 0).all()
    assert not np.array_equal(cases[0]["i_ovvv"], cases[1]["i_ovvv"])
    assert pool_gb > own_gb
