"""The device producer (libpt_rpt_inputs_df) on the GPU: its arrays against
the numpy restatement of tests/test_producer.py, and a restricted (T) solve
of the produced device arrays against the oracle on the restatement's."""
import numpy as np
import pytest

from libpt_b200 import ffi, synth
from oracle import oracle
from tests.test_gpu_parity import checker, close64
from tests.test_producer import df_inputs, random_factors

pytestmark = pytest.mark.gpu


def to_cuda(x):
    import torch
    return torch.as_tensor(np.ascontiguousarray(x)).to("cuda")


@pytest.mark.parametrize("o,v,naux", [(1, 1, 1), (3, 7, 12), (4, 11, 30),
                                      (5, 37, 64), (2, 70, 9)])
def test_produced_arrays_match_the_restatement(o, v, naux):
    b_oo, b_ov, b_vv, t2 = random_factors(o, v, naux, seed=o + v)
    got = ffi.rpt_inputs_df(to_cuda(b_oo), to_cuda(b_ov), to_cuda(b_vv),
                            to_cuda(t2))
    want = df_inputs(b_oo, b_ov, b_vv, t2)
    for name, ref in want.items():
        dev = got[name].cpu().numpy()
        assert dev.shape == ref.shape, name
        # cuBLAS sums the naux products in its own order: a few ulps of the
        # largest term
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(dev - ref).max() <= 1e-13 * scale, name
    # the amplitudes are moved, not computed: exact
    assert np.array_equal(got["t2"].cpu().numpy(), want["t2"])


def test_t2_in_place():
    """t2_abab may already sit in the abab half of the t2 output."""
    import torch
    o, v, naux = 3, 9, 10
    b_oo, b_ov, b_vv, t2 = random_factors(o, v, naux, seed=7)
    n2 = o * o * v * v
    t2_out = torch.empty(2 * n2, dtype=torch.float64, device="cuda")
    t2_out[n2:] = to_cuda(t2).reshape(-1)
    arrs = ffi.rpt_inputs_df(to_cuda(b_oo), to_cuda(b_ov), to_cuda(b_vv))
    code = ffi.lib().libpt_rpt_inputs_df(
        o, v, naux, to_cuda(b_oo).data_ptr(), to_cuda(b_ov).data_ptr(),
        to_cuda(b_vv).data_ptr(), t2_out.data_ptr() + 8 * n2,
        t2_out.data_ptr(), arrs["i_oovo"].data_ptr(),
        arrs["i_oovv"].data_ptr(), arrs["i_ovvv"].data_ptr(), None)
    torch.cuda.synchronize()
    assert code == ffi.LIBPT_OK
    assert np.array_equal(t2_out.cpu().numpy(),
                          df_inputs(b_oo, b_ov, b_vv, t2)["t2"])


@pytest.mark.parametrize("o,v,naux,fock", [(4, 20, 40, 0.0), (6, 31, 50, 1e-3)])
def test_solve_of_produced_inputs_matches_the_oracle(o, v, naux, fock):
    b_oo, b_ov, b_vv, t2 = random_factors(o, v, naux, seed=11 * o)
    case = synth.rpt_case(o, v, seed=o, fock=fock)    # d_ov, f_ov, t1
    host = dict(case)
    host.update(df_inputs(b_oo, b_ov, b_vv, t2))
    dev = {n: to_cuda(host[n]) for n in ("d_ov", "f_ov", "t1")}
    dev.update(ffi.rpt_inputs_df(to_cuda(b_oo), to_cuda(b_ov), to_cuda(b_vv),
                                 to_cuda(t2)))
    e = ffi.solve_device(case, dev)
    assert close64(e, oracle.solve(checker(), host))


def test_bad_arguments_are_refused():
    z = to_cuda(np.zeros(8))
    p = z.data_ptr()
    f = ffi.lib().libpt_rpt_inputs_df
    assert f(0, 2, 2, p, p, p, None, None, p, p, p, None) == ffi.LIBPT_ERR_ARG
    assert f(1, 1, 1, p, p, p, p, None, p, p, p, None) == ffi.LIBPT_ERR_ARG
    assert f(1, 1, 1, None, p, p, None, None, p, p, p, None) == ffi.LIBPT_ERR_ARG
    assert f(70000, 70000, 1, p, p, p, None, None, p, p, p, None) == \
        ffi.LIBPT_ERR_ARG


@pytest.mark.parametrize("oa,va,ob,vb,naux", [(3, 5, 2, 6, 7), (1, 1, 1, 2, 2),
                                              (2, 4, 0, 5, 3), (4, 13, 3, 14, 20),
                                              (2, 40, 3, 33, 17)])
def test_unrestricted_arrays_match_the_restatement(oa, va, ob, vb, naux):
    from tests.test_producer import df_inputs_u, spin_factors
    fa = spin_factors(oa, va, naux, seed=1)
    fb = spin_factors(ob, vb, naux, seed=2)
    got = ffi.upt_inputs_df([to_cuda(x) for x in fa], [to_cuda(x) for x in fb])
    want = df_inputs_u(fa, fb)
    for name, ref in want.items():
        dev = got[name].cpu().numpy()
        assert dev.shape == ref.shape, name
        scale = max(np.abs(ref).max() if ref.size else 0.0, 1e-300)
        assert np.abs(dev - ref).max(initial=0.0) <= 1e-13 * scale, name


@pytest.mark.parametrize("oa,va,ob,vb", [(4, 11, 3, 13), (5, 21, 4, 23)])
def test_unrestricted_solve_of_produced_inputs_matches_the_oracle(oa, va, ob,
                                                                  vb):
    from tests.test_producer import df_inputs_u, spin_factors
    naux = 30
    fa = spin_factors(oa, va, naux, seed=5)
    fb = spin_factors(ob, vb, naux, seed=6)
    case = synth.upt_case(oa, va, ob, vb, seed=oa, fock=1e-3)
    host = dict(case)
    host.update(df_inputs_u(fa, fb))
    dev = {n: to_cuda(host[n]) for n in ("d_ov", "f_ov", "t1", "t2")}
    dev.update(ffi.upt_inputs_df([to_cuda(x) for x in fa],
                                 [to_cuda(x) for x in fb]))
    e = ffi.solve_device(case, dev)
    assert close64(e, oracle.solve(checker(), host))
