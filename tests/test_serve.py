"""Serving loop, host side (no GPU): the device footprint that admission
uses (an exact sizing pass of the plan, libpt_footprint) and the server's
error reporting when no device is present."""
import ctypes

import pytest

from libpt_b200 import ffi

CASES = [("rpt", (4, 40)), ("upt", (4, 30, 3, 32)), ("rft", (4, 40)),
         ("uft", (3, 20, 4, 22))]
PRECS = [ffi.PREC_FP64, ffi.PREC_TF32X3, ffi.PREC_EMU64 | (6 << 8)]


@pytest.mark.parametrize("kind,sz", CASES)
@pytest.mark.parametrize("prec", PRECS)
def test_footprint_positive_and_ordered(kind, sz, prec):
    mp = prec == ffi.PREC_TF32X3
    f1 = ffi.footprint(kind, sz, mp=mp, precision=prec, round_triples=1)
    f2 = ffi.footprint(kind, sz, mp=mp, precision=prec, round_triples=2)
    fa = ffi.footprint(kind, sz, mp=mp, precision=prec)
    assert 0 < f1 < f2 <= fa
    # device inputs need no staging buffer
    fd = ffi.footprint(kind, sz, mp=mp, precision=prec, host=False,
                       round_triples=1)
    assert 0 < fd < f1


def test_footprint_grows_with_the_orbital_spaces():
    prev = 0
    for v in (20, 40, 80, 160):
        f = ffi.footprint("rpt", (6, v), round_triples=1)
        assert f > prev
        prev = f
    # the operands dominate: at least the padded OVVV and amplitude copies
    o, v = 6, 160
    assert f >= 8 * (o * v * v * v + 2 * o * o * v * v)


def test_footprint_emulated_adds_digit_planes():
    fp64 = ffi.footprint("rpt", (8, 96), round_triples=1)
    emu = ffi.footprint("rpt", (8, 96), precision=ffi.PREC_EMU64 | (6 << 8),
                        round_triples=1)
    # 6 one-byte planes per OVVV element on top of the FP64 copy
    assert emu > fp64 + 6 * 8 * 96 * 96 * 95 // 2


def test_footprint_rejects_bad_arguments():
    assert ffi.lib().libpt_footprint(7, 4, 4, 4, 4, 0, 0, 1, 0) == 0
    assert ffi.lib().libpt_footprint(0, 4, 4, 4, 4, 0, 9, 1, 0) == 0


def test_static_scratch_bound_matches_footprint():
    # libpt_rpt_dev_static accepts exactly what fits 64 MiB
    lim = 64 << 20
    assert ffi.footprint("rpt", (8, 64), host=False, round_triples=1) <= lim
    assert ffi.footprint("rpt", (12, 128), host=False, round_triples=1) > lim


def test_server_without_gpu_reports_an_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    code = ffi.lib().libpt_server_create(1 << 30, 4, ctypes.byref(h))
    assert code != ffi.LIBPT_OK and not h.value
    assert ffi.lib().libpt_last_error()
