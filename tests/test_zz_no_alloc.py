"""The allocation-free entry point libpt_rpt_dev_static.

It serves callers that cannot let a library allocate device memory (programs
whose device memory belongs to their own pool allocator, latency-sensitive
loops that must not synchronize the device through cudaMalloc/cudaFree).  The
test calls it through the C ABI twice in a row and compares each result with
the allocating device entry point libpt_rpt_dev, checks that the second call
leaves the device's free memory unchanged, and that a system too large for
the static scratch is rejected before any work.  This file is collected last
so that a failure here does not hide the results of the other tests.
"""
import ctypes

import numpy as np
import pytest

from libpt_b200 import ffi, synth

pytestmark = pytest.mark.gpu

ABS64, REL64 = 1e-9, 1e-12     # FP64 tolerance used by the parity tests


def _bind():
    L = ffi.lib()
    f = L.libpt_rpt_dev_static
    f.restype = ctypes.c_int
    f.argtypes = ([ctypes.c_size_t] * 2 + [ctypes.c_void_p] * 7
                  + [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)])
    return f


def _static_solve(f, case, t):
    e = ctypes.c_double(0.0)
    ptrs = [ctypes.c_void_p(t[n].data_ptr()) for n in ffi.PT_ARGS]
    rc = f(case["oa"], case["va"], *ptrs, None, ctypes.byref(e))
    return rc, e.value


def test_static_matches_allocating_entry_twice():
    import torch
    f = _bind()
    case = synth.rpt_case(8, 64, seed=42, fock=1e-3)   # the o=8, v=64 shape
    t = {n: torch.as_tensor(np.ascontiguousarray(case[n])).to(
        device="cuda", dtype=torch.float64) for n in ffi.PT_ARGS}
    e_ref = ffi.solve_device(case, t)
    rc1, e1 = _static_solve(f, case, t)
    assert rc1 == 0, ffi.lib().libpt_last_error()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    rc2, e2 = _static_solve(f, case, t)
    assert rc2 == 0, ffi.lib().libpt_last_error()
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    for e in (e1, e2):
        assert abs(e - e_ref) <= ABS64
        assert abs(e - e_ref) <= REL64 * abs(e_ref)
    assert free_after == free_before


@pytest.mark.parametrize("o,v", [(30, 300), (8, 78)])
def test_static_rejects_systems_beyond_its_scratch(o, v):
    """o=30, v=300 fails the cheap lower bound; o=8, v=78 passes it (35 MiB)
    but its exact footprint (67 MiB, sizing pass) exceeds the 64 MiB."""
    f = _bind()
    e = ctypes.c_double(0.0)
    # sizes are checked before any pointer is used; NULL pointers keep the
    # call harmless even if the check were missing
    rc = f(o, v, *([None] * 7), None, ctypes.byref(e))
    assert rc == 1
    assert b"scratch" in ffi.lib().libpt_last_error()


FRESH = r"""
import ctypes, sys
sys.path.insert(0, %r)
import numpy as np, torch
from libpt_b200 import ffi, synth
from tests.test_zz_no_alloc import _bind, _static_solve
torch.cuda.init()
case = synth.rpt_case(4, 20, seed=3)
t = {n: torch.as_tensor(np.ascontiguousarray(case[n])).to(
    device="cuda", dtype=torch.float64) for n in ffi.PT_ARGS}
torch.cuda.synchronize()
f = _bind()
free = [torch.cuda.mem_get_info()[0]]
for _ in range(2):
    rc, e = _static_solve(f, case, t)
    assert rc == 0, ffi.lib().libpt_last_error()
    torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info()[0])
print(free[0] - free[1], free[1] - free[2])
"""


def test_first_call_reserves_the_scratch_once():
    """In a fresh process: the first call on the device (which loads the
    library's device code) takes the static array's memory, at least
    LIBPT_STATIC_SCRATCH_BYTES; the second call takes none.  A caller whose
    pool allocator claims the device's memory makes its first call before
    creating the pool."""
    import os
    import subprocess
    import sys
    r = subprocess.run([sys.executable, "-c", FRESH % os.getcwd()],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    first, second = map(int, r.stdout.split()[-2:])
    assert first >= 64 << 20, first
    assert second == 0
