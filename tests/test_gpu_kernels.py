"""GPU self-tests of the contraction kernels (libpt_selftest): one job
C = A B1 - A B2 (two signed segments) on random operands against an FP64
product computed on the device, over ragged and tile-aligned shapes."""
import pytest

from libpt_b200 import ffi

pytestmark = pytest.mark.gpu

SHAPES = [(128, 256, 32), (1, 1, 1), (5, 7, 3), (200, 300, 100),
          (477, 1000, 477), (96, 130, 45), (300, 520, 700)]


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_dmma_fp64(m, n, k):
    assert ffi.selftest(ffi.PREC_FP64, m, n, k) < 1e-13


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_tcgen05_tf32x3(m, n, k):
    # 3xTF32 keeps ~21 bits per product and the tensor cores accumulate in
    # FP32: measured 2e-7 .. 1.1e-5 of max|C| for k <= 700
    assert ffi.selftest(ffi.PREC_TF32X3, m, n, k) < 5e-5


# emulated FP64: each 7-bit digit slice gains a factor 2^7 (measured:
# S=4 8e-9, S=5 6e-11, S=6 5e-13, S=7 5e-15 of max|C|)
EMU_BOUND = {4: 2e-8, 5: 2e-10, 6: 2e-12, 7: 2e-14}


@pytest.mark.parametrize("slices", [4, 5, 6, 7])
@pytest.mark.parametrize("m,n,k", SHAPES[1:])
def test_tcgen05_int8_emulated_fp64(slices, m, n, k):
    prec = ffi.PREC_EMU64 | (slices << 8)
    assert ffi.selftest(prec, m, n, k) < EMU_BOUND[slices]
