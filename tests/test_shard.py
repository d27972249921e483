"""Multi-GPU sharding of the matvec.

CPU: the shard assignment (host planner, plan-only init) covers the subtree
roots once, in contiguous balanced ranges; a world-size-2 gloo run sums the
ranks' partial results with the library's reduction (the partials come from
the oracle's subtree matvec over the boxes the library assigned).  GPU: the
shards' matvecs, run one after another on one GPU, sum to the unsharded
matvec and to the oracle.
"""
import os
import socket

import numpy as np
import pytest

from ifgf_b200 import workloads as W

from .helpers import densities_for, rel2


def _plan(n, nranks, rank, leaf=40, order=8):
    import ifgf_b200 as G

    pts = W.sphere_points(n, seed=0)
    op = G.HelmholtzIfgfOperator(20.0, leaf, order)
    op.set_shard(rank, nranks)
    op.init_plan_only(pts, pts)
    return op


@pytest.mark.parametrize("nranks", [2, 3, 5])
def test_shard_assignment_partitions_the_subtrees(nranks):
    n = 20000
    got = []
    level = None
    for r in range(nranks):
        lev, boxes = _plan(n, nranks, r).shard_boxes()
        level = lev if level is None else level
        assert lev == level and lev >= 1
        if len(boxes):
            assert np.all(np.diff(boxes) == 1)  # contiguous Morton range
        got.append(boxes)
    allb = np.concatenate(got)
    nb = _plan(n, 1, 0).num_boxes(level)
    assert np.array_equal(np.sort(allb), np.arange(nb))  # each root exactly once
    assert sum(len(b) > 0 for b in got) == min(nranks, nb)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, n, out_dir):
    import torch
    import torch.distributed as dist

    from ifgf_b200.distributed import reduce_partial
    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pts = W.sphere_points(n, seed=0)
        w = densities_for("helmholtz", n)
        op = _plan(n, world, rank)
        level, boxes = op.shard_boxes()
        o = O.OracleOperator("helmholtz", 20.0, 40, 8)
        o.init(pts, pts)
        part = o.mult_sample(w, level, boxes) if len(boxes) else np.zeros(n, complex)
        u = torch.from_numpy(np.ascontiguousarray(part))
        reduce_partial(u)
        np.save(os.path.join(out_dir, f"u{rank}.npy"), u.numpy())
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_sum_to_the_full_matvec(tmp_path):
    import torch.multiprocessing as mp

    from oracle import oracle as O

    n = 12000
    port = _free_port()
    mp.start_processes(_gloo_rank, args=(2, port, n, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    pts = W.sphere_points(n, seed=0)
    w = densities_for("helmholtz", n)
    o = O.OracleOperator("helmholtz", 20.0, 40, 8)
    o.init(pts, pts)
    full = o.mult(w)
    for r in range(2):
        u = np.load(tmp_path / f"u{r}.npy")
        assert rel2(u, full) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("name,nranks", [("helmholtz", 3), ("combined_field", 2), ("laplace", 4)])
def test_shards_sum_to_the_matvec_on_one_gpu(name, nranks):
    from oracle import oracle as O

    from .helpers import KERNELS, init_op, make_gpu_op, make_oracle_op

    n = 20000
    pts = W.sphere_points(n, seed=0)
    w = densities_for(name, n)
    full = make_gpu_op(name, leaf=50, order=8)
    init_op(full, name, pts, pts)
    uf = full.mult(w)
    parts = []
    for r in range(nranks):
        g = make_gpu_op(name, leaf=50, order=8)
        g.set_shard(r, nranks)
        init_op(g, name, pts, pts)
        parts.append(g.mult(w))
        assert g.stats()["missing_cone_lookups"] == 0
    assert rel2(sum(parts), uf) <= 1e-13
    o = make_oracle_op(name, leaf=50, order=8)
    init_op(o, name, pts, pts)
    assert rel2(sum(parts), o.mult(w)) <= 1e-12


@pytest.mark.gpu
def test_sharded_mixed_batches_sum_to_the_batch():
    # the path of bench.py --gpus N: every rank runs the batched mixed
    # pipeline (two plane groups here) over its subtrees
    from .helpers import make_gpu_op

    n = 20000
    pts = W.sphere_points(n, seed=0)
    w = np.stack([densities_for("helmholtz", n, seed=s) for s in range(5)])
    full = make_gpu_op("helmholtz", leaf=50, order=8)
    full.init(pts, pts)
    full.set_precision("mixed")
    uf = full.mult_batch(w)
    total = np.zeros_like(uf)
    for r in range(3):
        g = make_gpu_op("helmholtz", leaf=50, order=8)
        g.set_shard(r, 3)
        g.init(pts, pts)
        g.set_precision("mixed")
        total += g.mult_batch(w)
        assert g.stats()["missing_cone_lookups"] == 0
    for b in range(5):
        assert rel2(total[b], uf[b]) <= 1e-6, b


def test_plane_shares_partition_every_batch():
    from ifgf_b200.distributed import plane_range

    for world in range(1, 6):
        for n in range(0, 23):
            shares = [plane_range(n, r, world) for r in range(world)]
            assert shares[0][0] == 0 and shares[-1][1] == n
            for (a, b), (c, d) in zip(shares, shares[1:]):
                assert b == c  # contiguous, in rank order
            sizes = [b - a for a, b in shares]
            assert max(sizes) - min(sizes) <= 1


def _gloo_planes(rank, world, port, n, out_dir):
    import torch
    import torch.distributed as dist

    from ifgf_b200.distributed import PlaneParallel

    class Stub(PlaneParallel):
        # stands in for the GPU matvec: row p of the result is (1 + 2i) w_p + p
        def _apply_batch(self, w_rows, u_rows):
            lo, _ = self.share(n)
            rows = torch.arange(lo, lo + w_rows.shape[0], dtype=torch.float64)[:, None]
            u_rows[:] = (1 + 2j) * w_rows + rows

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = torch.from_numpy(np.stack([densities_for("helmholtz", 50, seed=s) for s in range(n)]))
        u = torch.zeros_like(w)
        pp = Stub(op=None)
        pp.mult_batch_device(w, u)
        pp.gather(u)
        np.save(os.path.join(out_dir, f"p{rank}.npy"), u.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 7), (3, 5)])
def test_gloo_plane_parallel_gathers_every_share(tmp_path, world, n):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_gloo_planes, args=(world, port, n, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    w = np.stack([densities_for("helmholtz", 50, seed=s) for s in range(n)])
    want = (1 + 2j) * w + np.arange(n)[:, None]
    for r in range(world):
        assert np.allclose(np.load(tmp_path / f"p{r}.npy"), want, rtol=0, atol=1e-12), r


@pytest.mark.gpu
def test_plane_parallel_and_sharded_batches_on_one_gpu():
    # one-rank NCCL group: both modes give the plain batched matvec
    import torch
    import torch.distributed as dist

    from ifgf_b200.distributed import PlaneParallel, ShardedOperator

    from .helpers import make_gpu_op

    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1)
    try:
        n = 6000
        pts = W.sphere_points(n, seed=0)
        w = np.stack([densities_for("helmholtz", n, seed=s) for s in range(5)])
        full = make_gpu_op("helmholtz", leaf=50, order=8)
        full.init(pts, pts)
        full.set_precision("mixed")
        # one upward kernel for both operators (each one's autotuner times its
        # own launches and may pick the other kernel on a near tie)
        full.set_upward_path("ffma")
        uf = full.mult_batch(w)
        dw = torch.from_numpy(w).cuda()
        du = torch.zeros_like(dw)
        pp = PlaneParallel(full)
        pp.mult_batch_device(dw, du)
        pp.gather(du)
        torch.cuda.synchronize()
        up = du.cpu().numpy()
        sh = ShardedOperator(make_gpu_op("helmholtz", leaf=50, order=8), pts, pts)
        sh.op.set_precision("mixed")
        sh.op.set_upward_path("ffma")
        ds = torch.zeros_like(dw)
        sh.mult_batch_device(dw, ds)
        torch.cuda.synchronize()
        us = ds.cpu().numpy()
        for b in range(5):
            assert rel2(up[b], uf[b]) <= 1e-14, b
            assert rel2(us[b], uf[b]) <= 1e-14, b
    finally:
        dist.destroy_process_group()
