"""A solve sharded over ranks, on one GPU: the ranks' runs are emulated one
after another on one plan (no kernel waits on another), their slot arrays
summed as the all-reduce would, and the energy compared bitwise with the
unsharded solve and, for the FP64 cases, with the oracle directly; then a
one-rank NCCL group runs the whole sharded path (libpt_b200.shard) through a
real all-reduce, checked against the oracle as well."""
import datetime
import os
import socket

import pytest

from libpt_b200 import ffi, synth
from oracle import oracle
from tests.test_gpu_parity import checker, close64, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,sz,prec", [
    ("rpt", (7, 33), ffi.PREC_FP64),
    ("upt", (4, 11, 3, 13), ffi.PREC_FP64),
    ("rft", (4, 10), ffi.PREC_FP64),
    ("uft", (3, 9, 4, 7), ffi.PREC_FP64),
    ("rpt", (8, 64), ffi.PREC_EMU64 | (6 << 8)),
    ("upt", (5, 21, 4, 23), ffi.PREC_EMU64 | (5 << 8)),
])
@pytest.mark.parametrize("size", [2, 3, 8])
def test_emulated_ranks_give_the_unsharded_energy(kind, sz, prec, size):
    import torch
    case = synth.make(kind, *sz, seed=5, fock=1e-3)
    plan = ffi.Plan(case, to_dev(case), precision=prec)
    try:
        plan.run()
        whole = plan.energy()
        acc = torch.zeros(plan.n, dtype=torch.float64, device="cuda")
        for r in range(size):
            plan.run_shard(r, size)
            torch.cuda.synchronize()
            own = plan.energy_slots().clone()
            mine = torch.as_tensor(ffi.shard_entries(plan.n, r, size),
                                   device="cuda")
            others = torch.ones(plan.n, dtype=torch.bool, device="cuda")
            others[mine] = False
            assert not own[others].any()       # only its own entries
            acc += own
        plan.energy_slots().copy_(acc)
        torch.cuda.synchronize()
        sharded = plan.energy()
        assert sharded == whole
        if prec == ffi.PREC_FP64:
            assert close64(sharded, oracle.solve(checker(), case))
    finally:
        plan.close()


def test_one_rank_nccl_group_runs_the_sharded_path():
    import torch
    import torch.distributed as dist
    from libpt_b200 import shard
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        case = synth.make("rpt", 6, 20, seed=9, fock=1e-3)
        e = shard.solve_sharded(case, to_dev(case))
        assert e == ffi.solve_host(case)
        assert close64(e, oracle.solve(checker(), case))
    finally:
        dist.destroy_process_group()
