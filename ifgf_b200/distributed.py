"""Multi-GPU matvec: one process per GPU under torch.distributed.

Every rank builds the operator on the full point sets with
``set_shard(rank, world)`` and applies its share of the source subtrees (a
contiguous Morton range of the subtrees rooted at the first level with far
pairs, balanced by modelled work); the partial target vectors are summed by
one all-reduce (NCCL over NVLink / NVSwitch on GPUs, gloo on CPU).  There is
no other exchange: the subtrees are independent because no box above the
shard level has far targets.
"""
import torch
import torch.distributed as dist

__all__ = ["reduce_partial", "ShardedOperator"]


def reduce_partial(u, group=None):
    """Sum the ranks' partial results in place (complex as real pairs)."""
    t = torch.view_as_real(u) if u.is_complex() else u
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return u


class ShardedOperator:
    """This rank's share of an IFGF operator.

    op: a constructed, not yet initialised operator (any kernel); the
    remaining arguments are those of its init.
    """

    def __init__(self, op, srcs, targets, normals=None, cutOff=None, group=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        op.set_shard(self.rank, self.world)
        if normals is None:
            op.init(srcs, targets, cutOff)
        else:
            op.init(srcs, targets, normals, cutOff)
        self.op = op

    @property
    def shard(self):
        """(level, boxes) of this rank's subtrees."""
        return self.op.shard_boxes()

    def mult_partial_device(self, w, u):
        """This rank's contribution A_r w into u (CUDA tensors), no collective."""
        stream = torch.cuda.current_stream(w.device).cuda_stream
        self.op.mult_device(w.data_ptr(), u.data_ptr(), stream)
        return u

    def mult_device(self, w, u):
        """u = A w, summed over the group (CUDA tensors on this rank's GPU)."""
        self.mult_partial_device(w, u)
        return reduce_partial(u, self.group)
