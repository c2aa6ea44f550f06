"""Serving loop on the GPU: continuous batching of uneven solves, admission
by footprint into a device pool, and the equality of every energy alone and
in the mix (bitwise: per-triple energies do not depend on which round or
launch ran a triple, and are summed in queue order)."""
import numpy as np
import pytest

from libpt_b200 import ffi, synth
from oracle import oracle
from tests.test_gpu_parity import checker, close64, to_dev

pytestmark = pytest.mark.gpu

EMU = ffi.PREC_EMU64 | (6 << 8)

MIX = [("rpt", (4, 20), 0), ("rpt", (6, 37), EMU), ("upt", (4, 11, 3, 13), 0),
       ("rft", (4, 10), 0), ("uft", (3, 9, 4, 7), EMU), ("rpt", (8, 64), 0),
       ("rpt", (5, 13), EMU), ("upt", (5, 21, 4, 23), EMU), ("rft", (5, 30), 0),
       ("rpt", (3, 2), 0), ("uft", (2, 5, 1, 4), 0), ("rpt", (7, 33), 0)]


def solo(case, prec):
    """The plan API on the same inputs, alone."""
    p = ffi.Plan(case, to_dev(case), precision=prec)
    p.run()
    e = p.energy()
    p.close()
    return e


@pytest.fixture(scope="module")
def mix_cases():
    return [(synth.make(k, *sz, seed=300 + i, fock=1e-3), prec)
            for i, (k, sz, prec) in enumerate(MIX)]


def test_mixed_stream_matches_solo_runs_bitwise(mix_cases):
    srv = ffi.Server(mem_budget=8 << 30)
    tickets = [srv.submit(c, precision=p) for c, p in mix_cases]
    got = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(mix_cases) and st["failed"] == 0
    assert st["rounds"] >= 1 and st["triples"] > 0
    for (c, p), (e, lat) in zip(mix_cases, got):
        assert e == solo(c, p), (c["kind"], p)
        assert lat > 0.0
    # and the FP64 ones against the oracle
    for (c, p), (e, _) in zip(mix_cases, got):
        if p == 0:
            assert close64(e, oracle.solve(checker(), c))


def test_alone_equals_in_the_mix(mix_cases):
    case, prec = mix_cases[5]                 # rpt (8, 64), FP64
    srv = ffi.Server(mem_budget=4 << 30)
    alone, _ = srv.wait(srv.submit(case, precision=prec))
    srv.close()
    srv = ffi.Server(mem_budget=4 << 30)
    tickets = []
    for i, (c, p) in enumerate(mix_cases):   # arrivals around it
        tickets.append(srv.submit(c, precision=p))
        if i == 3:
            mine = srv.submit(case, precision=prec)
    in_mix, _ = srv.wait(mine)
    for t in tickets:
        srv.wait(t)
    srv.close()
    assert in_mix == alone


def test_device_inputs_equal_host_inputs(mix_cases):
    case, prec = mix_cases[1]
    srv = ffi.Server(mem_budget=2 << 30)
    e_host, _ = srv.wait(srv.submit(case, precision=prec))
    t = to_dev(case)
    e_dev, _ = srv.wait(srv.submit(case, tensors=t, precision=prec))
    srv.close()
    assert e_host == e_dev


def test_admission_respects_the_budget(mix_cases):
    sizes = [ffi.footprint(c["kind"], [c[k] for k in ("oa", "va", "ob", "vb")
                                       if k in c], precision=p)
             for c, p in mix_cases]
    budget = 2 * max(sizes)
    srv = ffi.Server(mem_budget=budget, max_active=3)
    tickets = [srv.submit(c, precision=p) for c, p in mix_cases]
    energies = [srv.wait(t)[0] for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(mix_cases)
    assert st["peak_bytes_in_use"] <= st["pool_bytes"] <= budget + 256
    assert st["max_resident"] <= 3
    for (c, p), e in zip(mix_cases, energies):
        assert e == solo(c, p)


def test_oversized_solve_is_refused():
    case = synth.rpt_case(8, 64, seed=1)
    small = ffi.footprint("rpt", (8, 64)) // 2
    srv = ffi.Server(mem_budget=max(small, 1 << 20))
    t = srv.submit(case)
    with pytest.raises(ffi.LibptError, match="NOMEM"):
        srv.wait(t)
    srv.close()


def test_small_rounds_replay_graphs():
    cases = [synth.rpt_case(4, 16 + (i % 3), seed=i) for i in range(24)]
    srv = ffi.Server(mem_budget=2 << 30)
    ts = [srv.submit(c) for c in cases]
    es = [srv.wait(t)[0] for t in ts]
    st = srv.stats()
    srv.close()
    assert st["graph_rounds"] >= 1
    for c, e in zip(cases, es):
        assert e == solo(c, 0)


def test_large_rounds_replay_graphs():
    """Rounds of any size replay the graph of their variant set: every round
    but the first of each set is a replay, and the energies stay those of
    the plans alone."""
    # three solves of one size (one variant set), ~3.9e12 flops each: more
    # than two rounds each at the server's 1.5e12-flop rounds
    cases = [synth.rpt_case(12, 150, seed=40 + i) for i in range(3)]
    srv = ffi.Server(mem_budget=32 << 30, max_active=1)
    ts = [srv.submit(c) for c in cases]
    es = [srv.wait(t)[0] for t in ts]
    st = srv.stats()
    srv.close()
    assert st["rounds"] >= 6
    # a variant set is the GEMM variants plus which energy kernels run (the
    # same-spin triples come first in a queue, so a solve's rounds see a few
    # sets); only the first round of each set launches directly
    assert st["graph_rounds"] >= st["rounds"] - 4, st
    for c, e in zip(cases, es):
        assert e == solo(c, 0)
