"""Batches across ranks (svsim_b200.sharding): QAOA instances (size-balanced assignment)
and parameter points of one circuit (even split), with the gather of energies and
gradients, run as two gloo processes on the CPU.  The per-rank
evaluator is a deterministic stand-in (the GPU batch itself is covered by the gpu tests),
so these tests check the host logic: every instance evaluated exactly once, by the rank
the assignment names, and the gathered result equal to a single-process evaluation."""
import os
import socket

import numpy as np
import pytest

from svsim_b200 import circuits
from svsim_b200.sharding import ShardedAdjoint, ShardedQaoa, assign, split_even


class FakeEvaluator:
    """E_i = n_i + sum sin(gamma) + sum cos(beta); grad = (cos gamma, -sin beta)."""

    def __init__(self, instances):
        self.ns = np.array([inst.n for inst in instances], dtype=np.float64)

    def run(self, g, b):
        e = self.ns + np.sin(g).sum(axis=1) + np.cos(b).sum(axis=1)
        return e, np.concatenate([np.cos(g), -np.sin(b)], axis=1)


def test_assign_covers_every_instance_once_and_balances():
    insts = circuits.qaoa_instances(512)
    ns = [i.n for i in insts]
    for world in (1, 2, 3, 8):
        parts = assign(ns, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(insts)))
        loads = [sum(1 << ns[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= 1 << max(ns)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    insts = circuits.qaoa_instances(37, n_min=3, n_max=9, seed=11)
    seen = []

    def make_local(sub):
        seen.extend(inst.n for inst in sub)
        return FakeEvaluator(sub)

    sq = ShardedQaoa(insts, make_local=make_local)
    g = np.stack([i.gammas for i in insts])
    b = np.stack([i.betas for i in insts])
    e, grad = sq.run(g, b)
    np.savez(f"{out_path}.{rank}.npz", e=e, grad=grad, mine=np.array(sq.mine), seen=np.array(seen))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_run_two_gloo_ranks_matches_one_process(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn",
                       join=True)
    insts = circuits.qaoa_instances(37, n_min=3, n_max=9, seed=11)
    g = np.stack([i.gammas for i in insts])
    b = np.stack([i.betas for i in insts])
    e_ref, g_ref = FakeEvaluator(insts).run(g, b)
    parts = assign([i.n for i in insts], world)
    for r in range(world):
        d = np.load(f"{out}.{r}.npz")
        assert np.array_equal(d["e"], e_ref)
        assert np.array_equal(d["grad"], g_ref)
        assert list(d["mine"]) == parts[r]
        assert sorted(d["seen"]) == sorted(insts[i].n for i in parts[r])


def test_single_process_without_distributed():
    insts = circuits.qaoa_instances(5, n_min=3, n_max=6, seed=2)
    sq = ShardedQaoa(insts, make_local=FakeEvaluator)
    g = np.stack([i.gammas for i in insts])
    b = np.stack([i.betas for i in insts])
    e, grad = sq.run(g, b)
    e_ref, g_ref = FakeEvaluator(insts).run(g, b)
    assert sq.world == 1 and sq.mine == list(range(5))
    assert np.array_equal(e, e_ref) and np.array_equal(grad, g_ref)


# ---- parameter points of one circuit (ShardedAdjoint) -----------------------------------

class FakePoints:
    """E(p) = sum sin(p) + 0.5 sum p^2; grad = cos(p) + p; records the points it saw."""

    def __init__(self):
        self.seen = []

    def run(self, points, gradients=True):
        self.seen.extend(map(tuple, points))
        e = np.sin(points).sum(axis=1) + 0.5 * (points ** 2).sum(axis=1)
        return e, (np.cos(points) + points) if gradients else None


def _points(m=23, n_params=7, seed=5):
    return np.random.default_rng(seed).uniform(-np.pi, np.pi, size=(m, n_params))


def test_split_even_covers_each_point_once():
    for count in (0, 1, 5, 23, 64):
        for world in (1, 2, 3, 8):
            parts = split_even(count, world)
            assert len(parts) == world
            assert [i for p in parts for i in p] == list(range(count))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1


def _adj_worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    pc = circuits.hardware_efficient_ansatz(n=4, layers=1)
    fake = FakePoints()
    pts = _points(n_params=len(pc.params))
    sa = ShardedAdjoint(pc, None, make_local=lambda: fake)
    e, g = sa.run(pts)
    e2, g2 = sa.run(pts, gradients=False)
    np.savez(f"{out_path}.{rank}.npz", e=e, g=g, e2=e2, g2_none=np.array(g2 is None),
             seen=np.array(fake.seen))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_adjoint_two_gloo_ranks_matches_one_process(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    out = str(tmp_path / "adj")
    mp.start_processes(_adj_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn",
                       join=True)
    pc = circuits.hardware_efficient_ansatz(n=4, layers=1)
    pts = _points(n_params=len(pc.params))
    e_ref, g_ref = FakePoints().run(pts)
    parts = split_even(len(pts), world)
    for r in range(world):
        d = np.load(f"{out}.{r}.npz")
        assert np.array_equal(d["e"], e_ref) and np.array_equal(d["g"], g_ref)
        assert np.array_equal(d["e2"], e_ref) and bool(d["g2_none"])
        # each rank evaluated exactly its own run of points, once per call
        mine = pts[parts[r]]
        assert np.array_equal(d["seen"], np.concatenate([mine, mine]))


def test_sharded_adjoint_single_process():
    pc = circuits.hardware_efficient_ansatz(n=4, layers=1)
    pts = _points(m=3, n_params=len(pc.params))
    sa = ShardedAdjoint(pc, None, make_local=FakePoints)
    e, g = sa.run(pts)
    e_ref, g_ref = FakePoints().run(pts)
    assert sa.world == 1
    assert np.array_equal(e, e_ref) and np.array_equal(g, g_ref)
