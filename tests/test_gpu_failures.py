"""Failure detection, made to happen without faulting the GPU.

* Device-side waits: the bounded-wait probe (libpt_selftest_wait) loses a
  producer hand-off, so its consumer's mbarrier wait runs out after a short
  limit; the kernel records the timeout and returns, the call reports
  LIBPT_ERR_TIMEOUT, and the device stays usable (a contraction self-test
  passes right after).
* Host allocation: the reference's hooks (src/misc.c:22-47) -- a counting
  hook is actually called (and its blocks freed through the free hook); a
  hook that returns NULL makes the device-pointer API return
  LIBPT_ERR_NOMEM and the host API print its message and abort, the
  reference's err(1, ...) behaviour (src/pt.c:208-209) in a child process.
* Serving: a cancelled request ends with LIBPT_ERR_CANCELLED while queued
  or while running, returns its pool block, and leaves the other requests'
  energies bitwise those they have alone.
"""
import ctypes
import os
import signal
import subprocess
import sys
import time

import numpy as np
import pytest

from libpt_b200 import ffi, synth

pytestmark = pytest.mark.gpu


def test_lost_handoff_times_out_and_device_stays_usable():
    t0 = time.perf_counter()
    code, seen = ffi.selftest_wait(16, 5, 20.0)
    dt = time.perf_counter() - t0
    assert code == ffi.LIBPT_ERR_TIMEOUT
    assert seen == 5
    assert b"time limit" in ffi.lib().libpt_last_error()
    assert dt < 5.0
    code, seen = ffi.selftest_wait(16, 16, 20.0)
    assert code == ffi.LIBPT_OK and seen == 16
    assert ffi.selftest(ffi.PREC_FP64, 96, 128, 40) < 1e-14


def test_wait_probe_rejects_bad_arguments():
    assert ffi.selftest_wait(0, 0, 1.0)[0] == 1
    assert ffi.selftest_wait(8, 9, 1.0)[0] == 1
    assert ffi.selftest_wait(8, 4, 5000.0)[0] == 1


def test_allocation_hooks_are_called():
    libc = ctypes.CDLL(None)
    libc.malloc.restype = ctypes.c_void_p
    libc.malloc.argtypes = [ctypes.c_size_t]
    libc.free.argtypes = [ctypes.c_void_p]
    calls = {"malloc": 0, "free": 0}

    def my_malloc(n):
        calls["malloc"] += 1
        return libc.malloc(n)

    def my_free(p):
        calls["free"] += 1
        libc.free(p)

    case = synth.rpt_case(3, 9, seed=2)
    e0 = ffi.solve_host(case)
    ffi.set_host_allocator(my_malloc, my_free)
    try:
        e1 = ffi.solve_host(case)
    finally:
        ffi.set_host_allocator(None, None)
    assert e1 == e0
    assert calls["malloc"] >= 1 and calls["free"] == calls["malloc"]


def test_failing_allocation_hook_returns_nomem_on_device_api():
    import torch
    case = synth.rpt_case(3, 9, seed=2)
    dev = {n: torch.as_tensor(case[n]).to(device="cuda", dtype=torch.float64)
           for n in ffi.PT_ARGS}
    ffi.set_host_allocator(lambda n: None, None)
    try:
        with pytest.raises(ffi.LibptError) as ex:
            ffi.solve_device(case, dev)
    finally:
        ffi.set_host_allocator(None, None)
    assert ex.value.code == ffi.LIBPT_ERR_NOMEM
    assert ffi.solve_device(case, dev) == ffi.solve_host(case)


FAILING_HOOK = r"""
import sys
sys.path.insert(0, %r)
from libpt_b200 import ffi, synth
case = synth.rpt_case(3, 9, seed=2)
ffi.set_host_allocator(lambda n: None, None)
print("solving", flush=True)
ffi.solve_host(case)
print("returned", flush=True)
"""


def test_failing_allocation_hook_aborts_host_api():
    r = subprocess.run([sys.executable, "-c", FAILING_HOOK % os.getcwd()],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == -signal.SIGABRT, (r.returncode, r.stderr[-500:])
    assert "solving" in r.stdout and "returned" not in r.stdout
    assert "libpt_rpt: host allocation hook failed" in r.stderr


def _dev(case):
    import torch
    return {n: torch.as_tensor(np.ascontiguousarray(case[n])).to(
        device="cuda", dtype=torch.float64) for n in ffi.args_of(case["kind"])}


def test_cancelled_requests_end_and_others_are_unchanged():
    cases = [synth.make("rpt", 6, 40, seed=60 + i) for i in range(3)]
    # long (1.1e14 flops, seconds): cancelled while it runs
    cases.append(synth.make("rpt", 24, 200, seed=70))
    cases += [synth.make("upt", 5, 21, 4, 23, seed=80 + i) for i in range(3)]
    devs = [_dev(c) for c in cases]
    alone = [ffi.solve_device(c, d) for c, d in zip(cases, devs)]
    # max_active 1: the requests queue behind one another
    srv = ffi.Server(mem_budget=16 << 30, max_active=1)
    try:
        tk = [srv.submit(c, tensors=d) for c, d in zip(cases, devs)]
        srv.cancel(tk[5])                      # queued
        deadline = time.time() + 60
        while srv.stats()["completed"] < 3 and time.time() < deadline:
            time.sleep(0.005)
        srv.cancel(tk[3])                      # running (or about to)
        got = {}
        for i, t in enumerate(tk):
            try:
                got[i] = srv.wait(t)[0]
            except ffi.LibptError as ex:
                got[i] = ex.code
        st = srv.stats()
        times = srv.times(tk[0])
    finally:
        srv.close()
    assert got[5] == ffi.LIBPT_ERR_CANCELLED
    assert got[3] == ffi.LIBPT_ERR_CANCELLED
    for i in (0, 1, 2, 4, 6):
        assert got[i] == alone[i], i
    assert st["bytes_in_use"] == 0
    assert st["failed"] == 2
    assert len(times) == 4 and min(times) >= 0.0


def test_cancel_and_times_argument_errors():
    srv = ffi.Server(mem_budget=1 << 30)
    try:
        with pytest.raises(ffi.LibptError):
            srv.cancel(12345)
        case = synth.make("rpt", 3, 9, seed=1)
        t = srv.submit(case, tensors=_dev(case))
        e, lat = srv.wait(t)
        srv.cancel(t)                           # ended: keeps its result
        assert srv.wait(t)[0] == e
        q, prep, w, run = srv.times(t)
        assert abs((q + prep + w + run) - lat) <= 1e-6
    finally:
        srv.close()
