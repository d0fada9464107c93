"""z-slab sharding over torch.distributed ranks (mpdata_b200/sharded.py).

CPU tests: gloo ranks (world size 2-4, 127.0.0.1) each step their slab with
the CPU oracle as the per-rank solver; the gathered field must equal a
single-domain oracle run bit for bit, including plans whose halos span
several ranks.  The GPU test runs the real solver through the same path on
one rank (the exchange is empty) against the unsharded solver.
"""
import os
import socket

import numpy as np
import pytest

from mpdata_b200 import sharded, workloads


class OracleSlab:
    """The CPU oracle behind the per-rank solver interface (test infrastructure)."""

    def __init__(self, nx, ny, ns, order, opts):
        self.shape = (ns, ny, nx)
        self.order, self.opts = order, opts

    def set_faces(self, U, V, W):
        self.U, self.V, self.W = U.copy(), V.copy(), W.copy()

    def set_field(self, c):
        self.c = c.copy()

    def step(self, n):
        import oracle
        for _ in range(n):
            self.c = oracle.step_faces(self.U, self.V, self.W, self.c, self.order, **self.opts)

    def get_planes(self, k0, nk, out=None):
        if out is None:
            return self.c[k0:k0 + nk].copy()
        out[...] = self.c[k0:k0 + nk]
        return out

    def set_planes(self, k0, planes):
        self.c[k0:k0 + planes.shape[0]] = planes


def _case(nx, ny, ns, seed):
    import oracle
    case = workloads.random_case(nx, ny, ns, seed=seed)
    U, V, W = oracle.courant(case["dx"], case["dy"], case["ds"], case["dt"], case["u0"],
                             case["u1"], case["v0"], case["v1"], case["w0"], case["w1"],
                             dtype=np.float64)
    return [x.astype(np.float32) for x in (U, V, W, case["c0"])]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, shape, order, opts, steps, seed, outdir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                           world_size=world)
    try:
        nx, ny, ns = shape
        U, V, W, c = _case(nx, ny, ns, seed)
        s = sharded.ShardedSolver(nx, ny, ns, order=order, limiter=bool(opts.get("limiter")),
                                  make_solver=lambda a, b, c_: OracleSlab(a, b, c_, order, opts))
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(steps)
        full = s.gather(0)
        if rank == 0:
            np.save(os.path.join(outdir, "sharded.npy"), full)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,shape,order,opts,steps", [
    (2, (20, 14, 24), 2, {}, 3),
    (2, (20, 14, 24), 3, {"limiter": 1}, 3),
    (3, (17, 11, 30), 2, {"limiter": 1}, 4),
    (4, (16, 12, 14), 3, {"limiter": 1}, 2),   # halos of 5 planes span two owners
    (3, (15, 10, 12), 2, {"vv_fix": 1}, 3),
])
def test_sharded_equals_single_domain(tmp_path, world, shape, order, opts, steps):
    import oracle
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_rank_main, args=(world, port, shape, order, opts, steps, 11, str(tmp_path)),
             nprocs=world, join=True)
    got = np.load(tmp_path / "sharded.npy")
    U, V, W, c = _case(*shape, 11)
    ref = c
    for _ in range(steps):
        ref = oracle.step_faces(U, V, W, ref, order, **opts)
    assert np.array_equal(got, ref)


def test_plan_messages():
    p = sharded.SlabPlan(ns=14, world=4, halo=5)
    assert p.own == [(0, 4), (4, 8), (8, 11), (11, 14)]
    assert p.ext[2] == (3, 14)
    assert p.recvs(2) == [(0, 3, 4), (1, 4, 8), (3, 11, 14)]
    # every receive has its matching send, in the same order per peer
    for r in range(4):
        for peer, a, b in p.recvs(r):
            assert (r, a, b) in p.sends(peer)
    with pytest.raises(ValueError):
        sharded.SlabPlan(ns=4, world=5, halo=1)


@pytest.mark.gpu
def test_sharded_single_rank_gpu(tmp_path):
    """One rank over NCCL with the CUDA solver: the sharded path equals the
    plain solver bit for bit (the exchange is empty)."""
    import torch
    import torch.distributed as dist
    import mpdata_b200 as m
    port = _free_port()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        U, V, W, c = _case(70, 40, 30, 3)
        s = sharded.ShardedSolver(70, 40, 30, order=3, limiter=True, approx_div=True)
        s.set_faces(U, V, W)
        s.set_field(c)
        s.step(3)
        got = s.gather(0)
        with m.Solver(70, 40, 30, order=3, limiter=True, approx_div=True) as ref:
            ref.set_faces(U, V, W)
            ref.set_field(c)
            ref.step(3)
            assert np.array_equal(got, ref.get_field())
    finally:
        dist.destroy_process_group()
