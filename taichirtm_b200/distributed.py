"""Multi-GPU shot sharding: one process per GPU, shots partitioned across
ranks, one FP64 all-reduce of the stacked image (or gradient) at the end.

Shots are independent (the reference migrates them one per run and only sums
the images, examples/example_2nd_step.py:102-158, src/imaging.py:81-93), so
the data path needs no collective; the cross-shot sum is the only exchange.

Every rank takes the same collective steps in the same order, failures
included: a status all-reduce precedes the data reduction, so a rank whose
propagation failed (non-finite flag or an exception) makes every rank raise
instead of leaving the others waiting in the data collective."""
from typing import Callable, List, Sequence

import torch
import torch.distributed as dist


def shard_shots(costs: Sequence[float], world_size: int, rank: int) -> List[int]:
    """Indices of the shots given to ``rank``: longest-processing-time greedy
    on the per-shot cost (window cells x steps), ties by index; deterministic,
    so every rank computes the same partition without communicating."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world_size
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += float(costs[i])
    return [i for i in range(len(costs)) if owner[i] == rank]


def collective_device(group=None) -> torch.device:
    """The device the process group's collectives run on: this rank's current
    CUDA device under NCCL, the host under gloo.  Every collective of this
    module puts its tensors there, on the success and the failure path alike,
    so a failing rank never issues a collective that the others cannot
    match."""
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def reduce_result(local: torch.Tensor, status: int, group=None) -> torch.Tensor:
    """Sum ``local`` (an FP64 image/gradient stack) over ranks after agreeing
    that every rank succeeded.  Raises RuntimeError on every rank if any
    rank reported a non-zero status.  The status tensor lives on the group's
    collective device (``collective_device``), whatever ``local`` is, so a
    rank that failed before it had a result takes the same first step."""
    st = torch.tensor([int(status)], dtype=torch.int64, device=collective_device(group))
    dist.all_reduce(st, op=dist.ReduceOp.MAX, group=group)
    if int(st.item()) != 0:
        raise RuntimeError(f"a rank reported propagation status {int(st.item())}; result discarded")
    out = local.to(collective_device(group), torch.float64).clone()
    dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out.to(local.device)


def run_sharded(costs: Sequence[float], compute: Callable[[List[int]], torch.Tensor], group=None) -> torch.Tensor:
    """Partition shots, run ``compute(my_shot_indices)`` -> FP64 tensor on this
    rank, and return the sum over ranks.  An exception inside ``compute`` is
    turned into a non-zero status (so the other ranks do not hang) and
    re-raised after the status exchange."""
    ws = dist.get_world_size(group)
    rk = dist.get_rank(group)
    mine = shard_shots(costs, ws, rk)
    err = None
    try:
        local = compute(mine)
        status = 0
    except Exception as e:  # noqa: BLE001 - re-raised below after the collective
        err = e
        local = None
        status = 99
    if local is None:
        # same collective steps as the success path: the status all-reduce on
        # the group's device (reduce_result), after which every rank raises
        local = torch.zeros(1, dtype=torch.float64, device=collective_device(group))
    try:
        return reduce_result(local, status, group)
    except RuntimeError:
        if err is not None:
            raise err
        raise


def migrate_sharded(batched_factory, wavelets_of, observed_of, costs, isnap, group=None):
    """GPU helper: ``batched_factory(indices)`` -> BatchedRTM for those shots,
    ``wavelets_of``/``observed_of(indices)`` -> their input arrays.  Returns the
    FP64 stack summed over ranks."""
    def compute(idx):
        rtm = batched_factory(idx)
        try:
            ff, fb, stack = rtm.migrate(wavelets_of(idx), observed_of(idx), isnap=isnap)
            if int(max(ff.max(), fb.max())) != 0:
                raise FloatingPointError(f"propagation flags {ff.tolist()} / {fb.tolist()}")
            return stack
        finally:
            rtm.close()
    return run_sharded(costs, compute, group)
