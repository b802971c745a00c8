"""Replica parallelism for batches of samples (one process per GPU).

The state-vector path shards as independent units: every rank evaluates its own slice of the
encoder samples (or parameter sets) on its own GPU; no state is exchanged.  The only reduction
a training step needs is the sum of the ansatz gradients over samples
(``einsum('smp,sm->p')`` of mindquantum/framework/operations.py:145), a vector of P floats,
which ``allreduce_sum`` does with torch.distributed (NCCL across GPUs, gloo on CPU).
"""
import torch


def shard_bounds(n_items, rank, world):
    """[begin, end) of the contiguous slice of ``n_items`` owned by ``rank`` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} / world {world}")
    base, extra = divmod(n_items, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def shard(batch, rank, world):
    """The rows of ``batch`` (array or tensor, first axis = samples) owned by ``rank``."""
    b, e = shard_bounds(len(batch), rank, world)
    return batch[b:e]


def allreduce_sum(tensor, group=None):
    """Sum ``tensor`` over all ranks in place (no-op without an initialised process group)."""
    import torch.distributed as dist  # pylint: disable=import-outside-toplevel

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor


def ansatz_gradient(g_ans, dout, group=None):
    """Sum over samples of dout-weighted ansatz gradients, then over ranks.

    Args:
        g_ans: [n_samples][n_hams][n_ans] gradients of this rank's samples.
        dout: [n_samples][n_hams] incoming gradient of the expectations.
    """
    local = torch.einsum('smp,sm->p', torch.as_tensor(g_ans).real.double(), torch.as_tensor(dout).double())
    return allreduce_sum(local.contiguous(), group)
