"""bench.py's workload description: both arms print the same config, and its
flops are the reference's dgemm_ flops of the sampled triples (with stride 1,
the whole queue: rpt_flops(o, v), src/pt.c:49-158)."""
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
