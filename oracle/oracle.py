"""ctypes access to the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm import
this module, and only to check or time against the device library.

  restatement()  -> liboracle.so   (our C restatement, pt_oracle.c)
  reference()    -> _ref/libpt_ref.so (the reference compiled from its sources)

Both expose the pt.h signatures (src/pt.h:64-178); `solve()` calls either with
a case dict holding pt.h-layout numpy arrays.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

PT_ARGS = ("d_ov", "f_ov", "t1", "t2", "i_oovo", "i_oovv", "i_ovvv")
FT_ARGS = ("d_ov", "f2_ov", "l1", "t2", "l2", "i_oovv", "i2_t2f2_oovo",
           "i3_ovvv", "i6_oovo", "i7_ovvv")
KINDS = ("rpt", "upt", "rft", "uft")

_libs = {}


def _load(path, prefix):
    if path in _libs:
        return _libs[path]
    lib = ctypes.CDLL(path)
    for kind in KINDS:
        nsz = 2 if kind[0] == "r" else 4
        nptr = len(PT_ARGS) if kind[1:] == "pt" else len(FT_ARGS)
        for mp, ct in ((False, ctypes.c_double), (True, ctypes.c_float)):
            fn = getattr(lib, prefix + kind + ("_mp" if mp else ""))
            fn.restype = ctypes.c_double
            fn.argtypes = [ctypes.c_size_t] * nsz + [ctypes.POINTER(ct)] * nptr
    if prefix == "oracle_":
        lib.oracle_rpt_partials.restype = ctypes.c_size_t
        lib.oracle_rpt_partials.argtypes = (
            [ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t]
            + [ctypes.POINTER(ctypes.c_double)] * 8 + [ctypes.c_size_t])
    _libs[path] = (lib, prefix)
    return _libs[path]


def build(ref=True):
    """Compile the checkers; the reference build too when the environment
    names the reference's source directory (REFSRC) and it exists."""
    targets = ["oracle"]
    refsrc = os.environ.get("REFSRC", "")
    if ref and refsrc and os.path.isdir(refsrc):
        targets += ["ref", "REFSRC=" + refsrc]
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def restatement():
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        build(ref=False)
    return _load(path, "oracle_")


def reference_path():
    return os.path.join(HERE, "_ref", "libpt_ref.so")


def reference():
    path = reference_path()
    if not os.path.exists(path):
        raise FileNotFoundError(
            "reference build missing: run `make -C oracle ref` where the "
            "reference tree is present")
    return _load(path, "libpt_")


def args_of(kind):
    return PT_ARGS if kind[1:] == "pt" else FT_ARGS


def solve(which, case, mp=False):
    """Energy of `case` (dict: kind, oa, va, ob, vb, arrays) from a checker."""
    lib, prefix = which
    kind = case["kind"]
    dt = np.float32 if mp else np.float64
    ct = ctypes.c_float if mp else ctypes.c_double
    arrs = [np.ascontiguousarray(case[n], dtype=dt) for n in args_of(kind)]
    sizes = [int(case["oa"]), int(case["va"])]
    if kind[0] == "u":
        sizes += [int(case["ob"]), int(case["vb"])]
    fn = getattr(lib, prefix + kind + ("_mp" if mp else ""))
    return fn(*sizes, *[a.ctypes.data_as(ctypes.POINTER(ct)) for a in arrs])


def rpt_partials(case, kind):
    """Per-triple FP64 energies (kind 0: aaa, 1: aab) of a restricted case."""
    lib, _ = restatement()
    arrs = [np.ascontiguousarray(case[n], dtype=np.float64) for n in PT_ARGS]
    oa, va = int(case["oa"]), int(case["va"])
    p = ctypes.POINTER(ctypes.c_double)
    n = lib.oracle_rpt_partials(kind, oa, va, *[a.ctypes.data_as(p)
                                                for a in arrs], None, 0)
    out = np.zeros(max(n, 1))
    lib.oracle_rpt_partials(kind, oa, va, *[a.ctypes.data_as(p)
                                            for a in arrs],
                            out.ctypes.data_as(p), n)
    return out[:n]
