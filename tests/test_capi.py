"""CPU tests of the C ABI: the library builds, loads, and exports every
symbol include/pt.h declares; argument errors are reported without a GPU."""
import ctypes
import os
import re

import pytest

from libpt_b200 import build, ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    build.build()
    return ffi.lib()


def declared_functions():
    names = set()
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if not hdr.endswith(".h"):
            continue
        with open(os.path.join(ROOT, "include", hdr)) as fp:
            text = fp.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(libpt_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_reference_api():
    names = declared_functions()
    ref = ["libpt_print_banner", "libpt_set_malloc", "libpt_set_free",
           "libpt_rpt", "libpt_rpt_mp", "libpt_upt", "libpt_upt_mp",
           "libpt_rft", "libpt_rft_mp", "libpt_uft", "libpt_uft_mp"]
    for n in ref:
        assert n in names
    assert len(names) >= 27


def test_every_declared_symbol_is_exported(L):
    for n in declared_functions():
        assert hasattr(L, n), n


def test_banner_and_hooks(L, capfd):
    L.libpt_print_banner()
    out = capfd.readouterr().out
    assert "libpt" in out and len(out.strip().splitlines()) == 3
    L.libpt_set_malloc(None)
    L.libpt_set_free(None)


def test_argument_errors_need_no_gpu(L):
    h = ctypes.c_void_p()
    args = (ctypes.c_void_p * 7)()
    r = L.libpt_plan_create(9, 1, 1, 1, 1, args, 0, 0, None, ctypes.byref(h))
    assert r == 1 and not h.value
    assert b"kind" in L.libpt_last_error()
    r = L.libpt_plan_create(0, 2, 2, 2, 2, args, 0, 0, None, ctypes.byref(h))
    assert r == 1 and b"NULL" in L.libpt_last_error()
    r = L.libpt_plan_create(0, 2, 2, 2, 2, args, 0, 7, None, ctypes.byref(h))
    assert r == 1
    assert L.libpt_plan_queue_length(None) == -1
    e = ctypes.c_double()
    assert L.libpt_plan_energy(None, None, 0, ctypes.byref(e)) == 1
    assert L.libpt_plan_run(None, None, 0) == 1


def test_no_cpu_fallback_symbols(L):
    """The product library imports no BLAS and defines no CPU solver: its
    dynamic symbol table (nm -D) names neither dgemm_/sgemm_ nor oracle_*."""
    import subprocess
    out = subprocess.run(["nm", "-D", ffi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    for sym in ("dgemm_", "sgemm_", "oracle_"):
        assert sym not in out
