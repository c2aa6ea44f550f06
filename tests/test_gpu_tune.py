"""The autotuner (tune.cpp, plan.cu autotune): measured choices land in the
LIBPT_TUNE_FILE cache and are reused by a later process without measuring;
tuned, cached and untuned (LIBPT_AUTOTUNE=0) plans give the same energy
bitwise (tile shapes change which CTA computes an element, not its sum
order); a solve too small to repay its probes keeps the defaults."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SNIPPET = """
import sys
sys.path.insert(0, {root!r})
import torch
from libpt_b200 import ffi, synth
case = synth.make("rpt", {o}, {v}, seed=3, fock=1e-3)
dev = {{n: torch.as_tensor(case[n]).cuda() for n in ffi.args_of("rpt")}}
plan = ffi.Plan(case, dev, precision={prec})
plan.run()
print(repr(plan.energy()))
plan.close()
"""


def solve(o, v, prec, env_extra):
    env = dict(os.environ, LIBPT_TUNE_VERBOSE="1")
    env.pop("LIBPT_TUNE_FILE", None)
    env.pop("LIBPT_AUTOTUNE", None)
    env.update(env_extra)
    r = subprocess.run([sys.executable, "-c",
                        SNIPPET.format(root=ROOT, o=o, v=v, prec=prec)],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr
    return float(r.stdout.strip().splitlines()[-1]), r.stderr


@pytest.mark.parametrize("prec,marker", [(0, "DMMA tile rows"),
                                         (2 | (6 << 8), "INT8 tile")])
def test_tune_file_is_written_reused_and_energy_is_unchanged(tmp_path, prec,
                                                             marker):
    f = str(tmp_path / "tune.txt")
    e1, err1 = solve(20, 40, prec, {"LIBPT_TUNE_FILE": f})
    assert marker in err1
    lines = open(f).read().splitlines()
    assert len(lines) == 1 and lines[0].startswith(f"k0 o20,20 v40,40 p{prec & 0xFF}")
    e2, err2 = solve(20, 40, prec, {"LIBPT_TUNE_FILE": f})
    assert marker not in err2                      # cache hit: no probes
    assert open(f).read().splitlines() == lines    # nothing appended
    e3, err3 = solve(20, 40, prec, {"LIBPT_AUTOTUNE": "0"})
    assert marker not in err3
    assert e1 == e2 == e3


def test_small_solve_skips_the_probes(tmp_path):
    f = str(tmp_path / "tune.txt")
    e1, err = solve(4, 40, 0, {"LIBPT_TUNE_FILE": f})
    assert "skipped" in err and "DMMA tile rows" not in err
    assert not os.path.exists(f) or open(f).read() == ""
    e2, _ = solve(4, 40, 0, {"LIBPT_AUTOTUNE": "0"})
    assert e1 == e2
