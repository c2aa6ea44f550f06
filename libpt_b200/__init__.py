"""libpt_b200: perturbative-triples corrections (CCSD(T), EOM-CCSD(fT)) on
NVIDIA B200, behind the libpt C API (include/pt.h).

The compute path is the C/CUDA library libpt_b200/lib/libpt_b200.so; this
package is its Python mirror (ctypes) for tests, benchmarks and scripting:

    rpt(case) / upt / rft / uft      host-array entry points (libpt_rpt, ...)
    solve_device(case, tensors)      device-pointer twins (libpt_*_dev)
    Plan(case, tensors)              resident operands + triples queue

Importing the package does not load the library; the first call does, and
raises if it was not built.
"""
from . import synth
from .ffi import (FT_ARGS, PT_ARGS, LibptError, Plan, args_of, lib,
                  solve_device, solve_host)

__all__ = ["FT_ARGS", "PT_ARGS", "LibptError", "Plan", "args_of", "lib",
           "solve_device", "solve_host", "synth", "rpt", "upt", "rft", "uft"]


def _entry(kind):
    def f(case, mp=False):
        if case["kind"] != kind:
            raise ValueError(f"case kind {case['kind']} != {kind}")
        return solve_host(case, mp=mp)
    f.__name__ = kind
    f.__doc__ = f"Energy of a {kind} case through libpt_{kind}[_mp]."
    return f


rpt, upt, rft, uft = (_entry(k) for k in ("rpt", "upt", "rft", "uft"))
