"""One triples solve sharded over the ranks of a torch.distributed group.

The reference's MPI scheme (src/pt.c:197-221, 474-477) on GPUs: every rank
(one process per GPU) holds the full inputs, computes the triples q of the
queue with q % size == rank, and the ranks exchange once.  The reference
all-reduces one double; here the exchange is a sum all-reduce of the
per-triple energy slots (queue_length doubles, zero where another rank owns
the entry), after which every rank sums them in queue order and returns the
one-GPU energy bitwise.  NCCL moves the slots GPU to GPU (NVLink); with
gloo the same function runs on host tensors.
"""
import torch
import torch.distributed as dist

from . import ffi


def exchange_slots(slots, group=None):
    """Sum the ranks' energy-slot arrays in place.  Each entry is nonzero on
    its owner only, so the sum leaves every owner's value unchanged."""
    dist.all_reduce(slots, op=dist.ReduceOp.SUM, group=group)
    return slots


def solve_sharded(case, tensors, precision=ffi.PREC_FP64, mp=False,
                  group=None):
    """The energy of `case` (device tensors, the pt.h arguments) computed by
    all ranks of `group` together; every rank returns the same value."""
    rank, size = dist.get_rank(group), dist.get_world_size(group)
    plan = ffi.Plan(case, tensors, mp=mp, precision=precision)
    try:
        plan.run_shard(rank, size)
        torch.cuda.synchronize()      # the plan's stream has written its slots
        exchange_slots(plan.energy_slots(), group)
        torch.cuda.synchronize()
        return plan.energy()
    finally:
        plan.close()
