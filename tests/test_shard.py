"""Host logic of a solve sharded over ranks (src/pt.c:197-221, 474-477):
the ownership rule, the slot exchange over world-size-2 gloo ranks, and the
library's queue-order sum.  No GPU: the energies are seeded numbers standing
in for per-triple slots."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from libpt_b200 import ffi


def neumaier(x):
    s = c = 0.0
    for v in x:
        t = s + v
        c += (s - t) + v if abs(s) >= abs(v) else (v - t) + s
        s = t
    return s + c


@pytest.mark.parametrize("n,size", [(0, 1), (1, 1), (10, 3), (7, 8),
                                    (58740, 8), (1001, 2)])
def test_shard_entries_partition_the_queue(n, size):
    parts = [ffi.shard_entries(n, r, size) for r in range(size)]
    for r, p in enumerate(parts):
        assert np.all(p % size == r)          # src/pt.c:213
        assert np.all(np.diff(p) > 0)
    allq = np.sort(np.concatenate(parts))
    assert np.array_equal(allq, np.arange(n))
    counts = [len(p) for p in parts]
    assert max(counts) - min(counts) <= 1


@pytest.mark.parametrize("rank,size", [(-1, 2), (2, 2), (0, 0)])
def test_shard_entries_rejects_bad_rank(rank, size):
    with pytest.raises(ffi.LibptError):
        ffi.shard_entries(10, rank, size)


def test_energy_sum_is_compensated_queue_order_sum():
    rng = np.random.default_rng(3)
    e = rng.normal(0, 1e-4, 5000) * np.exp(rng.uniform(-20, 5, 5000))
    assert ffi.energy_sum(e) == neumaier(e)
    assert ffi.energy_sum([1e16, 1.0, -1e16]) == 1.0
    assert ffi.energy_sum([]) == 0.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, size, port, n, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=size,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from libpt_b200 import shard
        full = np.random.default_rng(11).normal(0, 1e-5, n)
        mine = ffi.shard_entries(n, rank, size)
        slots = torch.zeros(n, dtype=torch.float64)
        slots[torch.as_tensor(mine)] = torch.as_tensor(full[mine])
        shard.exchange_slots(slots)
        out[rank] = (slots.numpy().tobytes() == full.tobytes(),
                     ffi.energy_sum(slots.numpy()) == ffi.energy_sum(full))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size,n", [(2, 1237), (2, 1), (3, 400)])
def test_gloo_ranks_reassemble_the_one_rank_energy(size, n):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, size, port, n, out))
                 for r in range(size)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        assert [out[r] for r in range(size)] == [(True, True)] * size
