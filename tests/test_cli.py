"""pt_benchmark, the reference's benchmark command line (benchmark.c:348-392)
against this library.  CPU: argument handling (no solve runs).  GPU: every
type's energy equals the ctypes entry point's on the same random arrays."""
import os
import re
import subprocess

import numpy as np
import pytest

from libpt_b200 import build, ffi

CLI = build.CLI
TYPES = ["rpt", "upt", "rft", "uft", "rptmp", "uptmp", "rftmp", "uftmp"]


def run(*args, env=None):
    return subprocess.run([CLI, *map(str, args)], capture_output=True,
                          text=True, timeout=600, env=env)


def test_usage_and_bad_type():
    assert os.path.exists(CLI)
    r = run()
    assert r.returncode == 1 and "usage" in r.stderr
    r = run("ptr", 2, 3)
    assert r.returncode == 1 and "bad benchmark type" in r.stderr


def splitmix_uniform(start, n):
    """The CLI's generator (splitmix64, 53-bit uniforms) for draws
    start..start+n-1, vectorised."""
    with np.errstate(over="ignore"):
        i = np.arange(start + 1, start + n + 1, dtype=np.uint64)
        z = np.uint64(0x243f6a8885a308d3) + i * np.uint64(0x9e3779b97f4a7c15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
        z ^= z >> np.uint64(31)
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 2.0**53)


def cli_case(kind, oa, va, ob, vb):
    unr = kind[0] == "u"

    def size(c):
        if c == "ov":
            return oa * va + (ob * vb if unr else 0)
        if c == "oovv":
            return oa * oa * va * va + oa * ob * va * vb + (
                ob * ob * vb * vb + ob * oa * vb * va if unr else 0)
        if c == "oovo":
            return oa * oa * va * oa + oa * ob * va * ob + (
                ob * ob * vb * ob + ob * oa * vb * oa if unr else 0)
        return oa * va * (va * (va - 1) // 2) + oa * vb * va * vb + (
            ob * vb * (vb * (vb - 1) // 2) + ob * va * vb * va if unr else 0)

    pt = ["ov", "ov", "ov", "oovv", "oovo", "oovv", "ovvv"]
    ft = ["ov", "ov", "ov", "oovv", "oovv", "oovv", "oovo", "ovvv", "oovo",
          "ovvv"]
    classes = ft if kind[1:] == "ft" else pt
    case = dict(kind=kind, oa=oa, va=va, ob=ob, vb=vb)
    start = 0
    for name, c in zip(ffi.args_of(kind), classes):
        n = size(c)
        case[name] = splitmix_uniform(start, n) / 10000.0
        start += n
    return case


@pytest.mark.gpu
@pytest.mark.parametrize("t", TYPES)
def test_cli_energy_equals_entry_point(t):
    kind, mp = t[:3], t.endswith("mp")
    sz = (4, 13, 3, 11) if kind[0] == "u" else (5, 14, 5, 14)
    args = [t, sz[0], sz[1]] + ([sz[2], sz[3]] if kind[0] == "u" else [])
    r = run(*args)
    assert r.returncode == 0, r.stderr
    e = float(re.search(r"energy = (\S+)", r.stdout).group(1))
    case = cli_case(kind, *sz)
    assert e == ffi.solve_host(case, mp=mp)
    assert "done in" in r.stdout


@pytest.mark.gpu
def test_fp64_precision_environment_selects_emulated_fp64():
    import torch
    env = dict(os.environ, LIBPT_FP64_PRECISION="emu64:6")
    r = run("rpt", 5, 14, env=env)
    assert r.returncode == 0, r.stderr
    e = float(re.search(r"energy = (\S+)", r.stdout).group(1))
    case = cli_case("rpt", 5, 14, 5, 14)
    dev = {n: torch.as_tensor(case[n], device="cuda")
           for n in ffi.args_of("rpt")}
    plan = ffi.Plan(case, dev, precision=ffi.PREC_EMU64 | (6 << 8))
    try:
        plan.run()
        assert plan.slices == 6
        assert e == plan.energy()
    finally:
        plan.close()
