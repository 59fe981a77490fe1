"""Scale-out of one circuit over ranks (svsim_b200.scaleout).

* The planner on its own: its steps replayed on the whole state (segments by the oracle on
  physical positions, an exchange as the transposition of the top local bits with the
  rank bits) give the oracle's state bit for bit, for several rank counts.
* The distributed run: 2 and 4 gloo ranks on the CPU, each rank's chunk held in a CPU
  tensor with its segments applied by the oracle (a test stand-in for the GPU chunk),
  the exchange by torch.distributed.all_to_all_single; the gathered state and the
  samples against the oracle on the whole state.  The GPU chunk itself is covered by
  tests/test_gpu_scaleout.py.
"""
import os
import socket

import numpy as np
import pytest

from svsim_b200 import circuits, gates as G
from svsim_b200 import scaleout as S


def replay(plan, n, r, oracle):
    """The plan on the whole state: segments touch local positions only, so running them
    on the full vector is running them on every chunk."""
    m = n - r
    re = np.zeros(1 << n)
    im = np.zeros(1 << n)
    re[0] = 1.0
    idx = np.arange(1 << n, dtype=np.int64)
    for kind, g in plan.steps:
        if kind == "run":
            re, im = oracle.run(n, g, state=(re, im))
        else:
            src = idx.copy()
            for j in range(r):
                a, b = m - r + j, m + j
                ba, bb = (idx >> a) & 1, (idx >> b) & 1
                src = src & ~((1 << a) | (1 << b)) | (bb << a) | (ba << b)
            re, im = re[src], im[src]
    logical = np.zeros_like(idx)
    for q, p in enumerate(plan.final_pi):
        logical |= ((idx >> p) & 1) << q
    out_re, out_im = np.empty_like(re), np.empty_like(im)
    out_re[logical] = re
    out_im[logical] = im
    return out_re, out_im


def mixed_circuit(n, seed):
    rng = np.random.default_rng(seed)
    gl = G.from_array(circuits.random_matching_circuit(n, 3, seed=seed))
    gl += [G.CCX(n - 1, 0, n - 2), G.CRY(0.7, n - 1, 3), G.RZZ(0.4, 1, n - 2), G.SWAP(2, n - 1),
           G.CSWAP(n - 3, n - 1, 0), G.CU3(0.3, 0.2, 0.1, n - 2, n - 1), G.U3(*rng.uniform(0, 6, 3), n - 1)]
    return G.to_array(gl)


@pytest.mark.parametrize("n,r", [(8, 1), (9, 2), (10, 3), (12, 2)])
@pytest.mark.parametrize("restore", [True, False])
def test_plan_replayed_on_the_whole_state_matches_oracle(oracle, n, r, restore):
    g = mixed_circuit(n, seed=n + r)
    plan = S.plan_scaleout(g, n, r, restore=restore)
    m = n - r
    for kind, gates in plan.steps:
        if kind == "run":
            for rec in gates:
                assert all(q < m for q in S.gate_qubits(rec)), "a segment gate touches a rank bit"
    assert plan.n_exchanges >= 1
    if restore:
        assert plan.final_pi == list(range(n))
    re, im = replay(plan, n, r, oracle)
    ore, oim = oracle.run(n, g)
    assert np.array_equal(re, ore) and np.array_equal(im, oim)


def test_plan_rejects_what_cannot_be_placed():
    with pytest.raises(ValueError):
        S.plan_scaleout(G.to_array([G.H(0)]), 4, 3)
    with pytest.raises(ValueError):
        S.plan_scaleout(G.to_array([G.C4X(0, 1, 2, 3, 5)]), 7, 2)


class CpuChunk:
    """Test stand-in for GpuChunk: the chunk in a CPU tensor, segments by the oracle."""

    def __init__(self, m, oracle):
        import torch
        self.m, self.o, self.device = m, oracle, None
        self.view = torch.zeros(2 << m, dtype=torch.float64)
        self.scratch = torch.empty_like(self.view)

    def state(self):
        v = self.view.numpy()
        return v[0::2].copy(), v[1::2].copy()

    def run(self, gates):
        import torch
        re, im = self.o.run(self.m, gates, state=self.state())
        self.view[0::2] = torch.from_numpy(re)
        self.view[1::2] = torch.from_numpy(im)

    def sync(self):
        pass

    def reset(self, rank):
        self.view.zero_()
        if rank == 0:
            self.view[0] = 1.0

    def measure(self, u):
        re, im = self.state()
        return self.o.measure(self.m, re, im, u)

    def norm2(self):
        return float((self.view * self.view).sum())

    def close(self):
        pass


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, out_path):
    import datetime
    import torch.distributed as dist
    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    r = world.bit_length() - 1
    sim = S.ScaleOutSimulation(n, chunk=CpuChunk(n - r, Oracle()))
    g = mixed_circuit(n, seed=3 * n + world)
    plan = sim.run(g[: len(g) // 2])             # two calls: the layout carries over
    plan2 = sim.run(g[len(g) // 2:])
    got = sim.gather_state()
    u = np.random.default_rng(5).random(512)
    samples = sim.measure(u)
    if rank == 0:
        np.savez(out_path, re=got[0], im=got[1], samples=samples,
                 exchanges=plan.n_exchanges + plan2.n_exchanges)
    else:
        np.savez(f"{out_path}.{rank}.npz", samples=samples)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_distributed_run_matches_oracle(oracle, tmp_path, world):
    import torch.multiprocessing as mp
    n = 10
    out = str(tmp_path / "res.npz")
    mp.start_processes(_worker, args=(world, _free_port(), n, out), nprocs=world, start_method="spawn",
                       join=True)
    d = np.load(out)
    g = mixed_circuit(n, seed=3 * n + world)
    ore, oim = oracle.run(n, g)
    assert np.array_equal(d["re"], ore) and np.array_equal(d["im"], oim)
    assert int(d["exchanges"]) >= 1
    u = np.random.default_rng(5).random(512)
    ref, _ = oracle.measure(n, ore, oim, u)
    assert np.array_equal(d["samples"], ref)
    for rk in range(1, world):
        assert np.array_equal(np.load(f"{out}.{rk}.npz")["samples"], ref)
