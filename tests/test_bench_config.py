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


def test_cpu_extrapolation_is_the_workload_flops_over_the_rate():
    a = args_of()
    x = bench.extrapolation(a, 0.08)
    assert abs(x["extrapolated_solve_seconds"] -
               bench.rpt_flops(45, 477) / 0.08e12) < 1e-6
    assert x["extrapolation"].startswith("extrapolated: rpt o=45 v=477")


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
    names = [f[0] for f in bench.precision_forms(ffi)]
    assert names == ["fp64", "emu64_s4", "emu64_s5", "emu64_s6", "emu64_s7",
                     "emu64_auto", "tf32x3"]
    assert [f[2] for f in bench.precision_forms(ffi)].count(True) == 1
