"""Batched QAOA over several GPUs, one process per GPU.

The instances of a batch are independent, so they are split across the ranks by size
(longest-processing-time order on 2^n, which is what one evaluation's time and memory
follow), each rank evaluates its own share on its own GPU in one batched launch
(svb_qaoa_*), and the energies and gradients are gathered with one all-reduce over
disjoint slots (every other slot adds an exact zero).  There is no collective on the data
path and no rank reads another GPU's memory.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def assign(n_qubits: Sequence[int], world: int) -> list[list[int]]:
    """Instance indices per rank: largest instances first, each to the rank with the
    smallest load so far (ties to the lower rank); indices ascending within a rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(n_qubits)), key=lambda i: (-(1 << int(n_qubits[i])), i))
    loads = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        out[r].append(i)
        loads[r] += 1 << int(n_qubits[i])
    return [sorted(x) for x in out]


class ShardedQaoa:
    """Energy and gradient of every instance of a batch, evaluated across the ranks of
    `group` (torch.distributed; a single process when it is not initialised).

    `make_local(instances)` builds this rank's evaluator; by default a
    ``_native.QaoaBatch`` on `device`.  Its ``run(gammas, betas)`` returns
    ``(energies [m], grads [m, 2p])`` for its m instances."""

    def __init__(self, instances, device: int = 0, precision: int | None = None,
                 group=None, make_local: Callable | None = None):
        import torch.distributed as dist
        self.distributed = dist.is_available() and dist.is_initialized()
        self.group = group
        self.world = dist.get_world_size(group) if self.distributed else 1
        self.rank = dist.get_rank(group) if self.distributed else 0
        self.n_inst = len(instances)
        self.p = len(instances[0].gammas)
        self.parts = assign([inst.n for inst in instances], self.world)
        self.mine = self.parts[self.rank]
        if make_local is None:
            from . import _native as nat
            prec = nat.SVB_FP64 if precision is None else precision

            def make_local(sub):
                return nat.QaoaBatch(sub, device, prec)
        self.local = make_local([instances[i] for i in self.mine]) if self.mine else None
        self.device = device

    def run(self, gammas, betas):
        """gammas, betas: [n_instances, p] (the same on every rank).  Returns the full
        (energies [n], grads [n, 2p]) on every rank."""
        g = np.asarray(gammas, dtype=np.float64).reshape(self.n_inst, self.p)
        b = np.asarray(betas, dtype=np.float64).reshape(self.n_inst, self.p)
        full = np.zeros((self.n_inst, 1 + 2 * self.p))
        if self.local is not None:
            idx = np.asarray(self.mine)
            e, grad = self.local.run(g[idx], b[idx])
            full[idx, 0] = e
            full[idx, 1:] = grad
        if self.world > 1:
            import torch
            import torch.distributed as dist
            on_gpu = dist.get_backend(self.group) == "nccl"
            t = torch.from_numpy(full)
            if on_gpu:
                t = t.to(f"cuda:{self.device}")
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
            full = t.cpu().numpy()
        return full[:, 0].copy(), full[:, 1:].copy()

    def close(self):
        if self.local is not None and hasattr(self.local, "close"):
            self.local.close()
        self.local = None
