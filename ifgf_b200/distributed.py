"""Multi-GPU matvec: one process per GPU under torch.distributed.

Two ways to spread the work:

* ``ShardedOperator`` -- one matvec over several GPUs.  Every rank builds the
  operator on the full point sets with ``set_shard(rank, world)`` and applies
  its share of the source subtrees (a contiguous Morton range of the subtrees
  rooted at the first level with far pairs, balanced by modelled work); the
  partial target vectors are summed by one all-reduce (NCCL over NVLink /
  NVSwitch on GPUs, gloo on CPU).  There is no other exchange: the subtrees
  are independent because no box above the shard level has far targets.
* ``PlaneParallel`` -- many matvecs (a batch of right-hand sides, or the
  wavenumbers of a frequency set): every rank holds the whole operator and
  applies it to a contiguous share of the planes.  No exchange on the data
  path; ``gather`` assembles the full result on every rank when wanted.
"""
import torch
import torch.distributed as dist

__all__ = ["reduce_partial", "ShardedOperator", "plane_range", "PlaneParallel"]


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

    def mult_batch_device(self, w, u):
        """Every row of w (batch, N) -> u (batch, M), summed over the group."""
        stream = torch.cuda.current_stream(w.device).cuda_stream
        self.op.mult_batch_device(w.data_ptr(), u.data_ptr(), w.shape[0], stream)
        return reduce_partial(u, self.group)

    def mult_wavenumbers_device(self, ks, w, u):
        """Row p of u = A(k_p) w_p, summed over the group."""
        stream = torch.cuda.current_stream(w.device).cuda_stream
        self.op.mult_wavenumbers_device(ks, w.data_ptr(), u.data_ptr(), stream)
        return reduce_partial(u, self.group)


def plane_range(n, rank, world):
    """Contiguous share [lo, hi) of n planes for `rank` of `world` ranks (the
    first n % world ranks take one more)."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


class PlaneParallel:
    """Batches split over ranks: every rank holds the whole, initialised
    operator `op` and applies it to its contiguous share of the planes
    (right-hand sides or wavenumbers); nothing is exchanged on the data path.
    """

    def __init__(self, op, group=None):
        self.op = op
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def share(self, n):
        return plane_range(n, self.rank, self.world)

    def _apply_batch(self, w_rows, u_rows):
        stream = torch.cuda.current_stream(w_rows.device).cuda_stream
        self.op.mult_batch_device(w_rows.data_ptr(), u_rows.data_ptr(), w_rows.shape[0], stream)

    def _apply_wavenumbers(self, ks, w_rows, u_rows):
        stream = torch.cuda.current_stream(w_rows.device).cuda_stream
        self.op.mult_wavenumbers_device(ks, w_rows.data_ptr(), u_rows.data_ptr(), stream)

    def mult_batch_device(self, w, u):
        """u[lo:hi] = A w[lo:hi] for this rank's share (w: (n, N), u: (n, M),
        contiguous); the other rows of u are left as they are."""
        lo, hi = self.share(w.shape[0])
        if hi > lo:
            self._apply_batch(w[lo:hi], u[lo:hi])
        return u

    def mult_wavenumbers_device(self, ks, w, u):
        """u[p] = A(k_p) w[p] for this rank's share of the wavenumbers."""
        lo, hi = self.share(w.shape[0])
        if hi > lo:
            self._apply_wavenumbers(list(ks)[lo:hi], w[lo:hi], u[lo:hi])
        return u

    def gather(self, u):
        """Fill every rank's u (n, M) with all ranks' shares (one
        all-gather of equal-sized, zero-padded shares)."""
        n = u.shape[0]
        lo, hi = self.share(n)
        width = -(-n // self.world)
        t = torch.view_as_real(u) if u.is_complex() else u
        mine = torch.zeros((width,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
        mine[: hi - lo] = t[lo:hi]
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        dist.all_gather(parts, mine, group=self.group)
        for r, part in enumerate(parts):
            a, b = plane_range(n, r, self.world)
            t[a:b] = part[: b - a]
        return u
