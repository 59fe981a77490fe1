"""Scale-out of one circuit (svsim_b200.scaleout) on the GPU chunk backend.

One GPU per test run here, so the ranks of a 2- and 4-rank layout are held as GpuChunk
objects in one process: every segment runs on each chunk through the engines, and the
exchange step is done in-process on the chunks' zero-copy device views with the same
transposition all_to_all_single performs (block j of chunk i <-> block i of chunk j).  No
collective runs and no kernel waits on another.  The ScaleOutSimulation class itself runs
over a one-rank NCCL group.  All against the oracle on the whole state."""
import os
import socket

import numpy as np
import pytest

from svsim_b200 import circuits, gates as G
from svsim_b200 import scaleout as S

pytestmark = pytest.mark.gpu


def circuit(n, seed):
    gl = G.from_array(circuits.random_matching_circuit(n, 4, seed=seed))
    gl += [G.CCX(n - 1, 0, n - 2), G.CRY(0.7, n - 1, 3), G.RZZ(0.4, 1, n - 2), G.SWAP(2, n - 1),
           G.CSWAP(n - 3, n - 1, 0), G.CU3(0.3, 0.2, 0.1, n - 2, n - 1)]
    return G.to_array(gl)


@pytest.mark.parametrize("n,r", [(14, 1), (16, 2)])
def test_gpu_chunks_with_in_process_exchange(oracle, n, r):
    import torch
    from svsim_b200 import _native as nat
    R, m = 1 << r, n - r
    chunks = [S.GpuChunk(m, 0, nat.SVB_FP64) for _ in range(R)]
    for rk, c in enumerate(chunks):
        c.reset(rk)
    g = circuit(n, seed=n)
    plan = S.plan_scaleout(g, n, r)
    assert plan.n_exchanges >= 1
    for kind, gates in plan.steps:
        if kind == "run":
            for c in chunks:
                c.run(gates)
        else:
            for c in chunks:
                c.sync()
            blocks = [c.view.view(R, -1).clone() for c in chunks]
            for i, c in enumerate(chunks):
                for j in range(R):
                    c.view.view(R, -1)[j].copy_(blocks[j][i])
            torch.cuda.synchronize()
    states = [c.state() for c in chunks]
    re = np.concatenate([s[0] for s in states])
    im = np.concatenate([s[1] for s in states])
    ore, oim = oracle.run(n, g)
    assert np.max(np.abs(re - ore)) <= 1e-12 and np.max(np.abs(im - oim)) <= 1e-12
    for c in chunks:
        c.close()


def test_scaleout_simulation_one_rank_nccl(oracle):
    import datetime
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=__import__("torch").device("cuda:0"))
    try:
        n = 14
        sim = S.ScaleOutSimulation(n, device=0)
        g = circuit(n, seed=7)
        sim.run(g)
        re, im = sim.gather_state()
        ore, oim = oracle.run(n, g)
        assert np.max(np.abs(re - ore)) <= 1e-12 and np.max(np.abs(im - oim)) <= 1e-12
        u = np.random.default_rng(2).random(256)
        ref, _ = oracle.measure(n, ore, oim, u)
        assert np.array_equal(sim.measure(u), ref)
        sim.close()
    finally:
        dist.destroy_process_group()
