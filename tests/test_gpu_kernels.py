"""GPU self-tests of the contraction kernels (libpt_selftest): one job
C = A B1 - A B2 (two signed segments) on random operands against an FP64
product computed on the device, over ragged and tile-aligned shapes."""
import pytest

from libpt_b200 import ffi

pytestmark = pytest.mark.gpu

SHAPES = [(128, 256, 32), (1, 1, 1), (5, 7, 3), (200, 300, 100),
          (477, 1000, 477), (96, 130, 45), (300, 520, 700)]


@pytest.mark.parametrize("variant", [0, 1])       # 128-row, 96-row tiles
@pytest.mark.parametrize("m,n,k", SHAPES)
def test_dmma_fp64(m, n, k, variant):
    assert ffi.selftest(ffi.PREC_FP64, m, n, k, variant) < 1e-14


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_tcgen05_tf32x3(m, n, k):
    # 3xTF32 keeps ~21 bits per product and the tensor cores accumulate in
    # FP32 (truncating): about 1.6e-8 per accumulation step
    assert ffi.selftest(ffi.PREC_TF32X3, m, n, k) < 5e-5


# emulated FP64: each 7-bit digit slice gains a factor 2^7.  The S(S+1)/2
# kept digit products leave (S+1) 2^(-7S-2) of |a||b| per product and each
# operand's truncation 2^(-7S-1); with row / column scales up to 4x the
# values, the error over sum |a||b| stays below 2^(-7S+6)
EMU_BOUND = {s: 2.0 ** (-7 * s + 6) for s in (4, 5, 6, 7)}
# 8-bit balanced digits (a 7-bit top digit, 8 bits per lower digit): each
# operand's truncation 2^(-8S) instead of 2^(-7S-1), the same terms besides
EMU8_BOUND = {s: 2.0 ** (-8 * s + 8) for s in (4, 5, 6)}


# every compiled INT8 tile variant (tile width x K chunk; one CTA, a CTA
# pair, or A read from TMEM) of each slice count
I8_VARIANTS = {4: 4, 5: 4, 6: 3, 7: 1}


@pytest.mark.parametrize("slices,variant",
                         [(s, t) for s, n in I8_VARIANTS.items()
                          for t in range(n)])
@pytest.mark.parametrize("m,n,k", SHAPES[1:])
def test_tcgen05_int8_emulated_fp64(slices, variant, m, n, k):
    prec = ffi.PREC_EMU64 | (slices << 8)
    assert ffi.selftest_variants(prec) == I8_VARIANTS[slices]
    assert ffi.selftest(prec, m, n, k, variant) < EMU_BOUND[slices]


@pytest.mark.parametrize("slices,variant",
                         [(s, t) for s, n in I8_VARIANTS.items() if s <= 6
                          for t in range(n)])
@pytest.mark.parametrize("m,n,k", SHAPES[1:])
def test_tcgen05_int8_emulated_fp64_8bit_digits(slices, variant, m, n, k):
    """8-bit balanced digit planes (carries into the digit above)."""
    prec = ffi.PREC_EMU64 | (slices << 8)
    e8 = ffi.selftest(prec, m, n, k, variant, dbits=8)
    assert e8 < EMU8_BOUND[slices]
    if slices <= 5 and m * n >= 10000:   # the extra bit per plane shows
        assert e8 < ffi.selftest(prec, m, n, k, variant)


@pytest.mark.parametrize("m,n,k", [(5, 7, 3), (300, 520, 700)])
def test_device_memory_tensor_maps(m, n, k):
    """The form batched multi-solve launches use: tensor maps read from
    device memory (fenced per CTA) instead of kernel parameters."""
    assert ffi.selftest(ffi.PREC_FP64, m, n, k, 0, device_maps=True) < 1e-14
    assert ffi.selftest(ffi.PREC_TF32X3, m, n, k, device_maps=True) < 5e-5
    for s in (4, 6):
        prec = ffi.PREC_EMU64 | (s << 8)
        assert ffi.selftest(prec, m, n, k, 0, device_maps=True) < EMU_BOUND[s]
        assert ffi.selftest(prec, m, n, k, 0, device_maps=True,
                            dbits=8) < EMU8_BOUND[s]


@pytest.mark.parametrize("lo,hi", [(-10, 10), (-1000, 1000)])
def test_energy_reciprocal_is_within_two_ulp_of_division(lo, hi):
    """The energy epilogues multiply by a Newton-refined reciprocal of the
    denominator instead of dividing: within 2 ulp of IEEE 1.0 / d over the
    range their docs state (the (T) denominators lie near 2^-3..2^5)."""
    assert ffi.selftest_recip(lo, hi, 1 << 22) <= 2.0


def test_energy_reciprocal_rejects_bad_ranges():
    with pytest.raises(ffi.LibptError):
        ffi.selftest_recip(-1001, 0, 16)
    with pytest.raises(ffi.LibptError):
        ffi.selftest_recip(3, 2, 16)
