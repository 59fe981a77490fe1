"""Batched work over several GPUs, one process per GPU.

Two kinds of batch shard with no exchange on the data path:

* QAOA instances (ShardedQaoa).  The instances are split across the ranks by size
  (longest-processing-time order on 2^n, which is what one evaluation's time and memory
  follow); each rank evaluates its share on its own GPU in one batched launch
  (svb_qaoa_*).
* Parameter points of one parametrised circuit (ShardedAdjoint): a batch of parameter
  sets, or the shifted points of finite differences or the parameter-shift rule.  Every
  point costs the same, so the points are split into equal contiguous runs; each rank
  computes the energy (and the adjoint gradient, svb_adjoint) of its points on its GPU.

In both, the results are gathered with one all-reduce over disjoint rows (every other
rank adds an exact zero), and no rank reads another GPU's memory.
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


def split_even(count: int, world: int) -> list[list[int]]:
    """Indices 0..count-1 in `world` contiguous runs whose sizes differ by at most one
    (the first count % world runs get the extra index)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(count, world)
    out, start = [], 0
    for r in range(world):
        size = base + (1 if r < extra else 0)
        out.append(list(range(start, start + size)))
        start += size
    return out


def _gather_rows(full: np.ndarray, world: int, group, device: int) -> np.ndarray:
    """Sums the ranks' row blocks (each rank filled only its own rows) on every rank."""
    if world == 1:
        return full
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(full)
    if dist.get_backend(group) == "nccl":
        t = t.to(f"cuda:{device}")
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


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
        full = _gather_rows(full, self.world, self.group, self.device)
        return full[:, 0].copy(), full[:, 1:].copy()

    def close(self):
        if self.local is not None and hasattr(self.local, "close"):
            self.local.close()
        self.local = None


class AdjointPoints:
    """One rank's evaluator of ShardedAdjoint: an FP64 handle on `device` that runs the
    circuit at each point (svb_adjoint for energy and gradient, or svb_run and
    svb_expectation for the energy alone)."""

    def __init__(self, circuit, terms, device: int = 0):
        from . import _native as nat
        self.circuit = circuit
        self.terms = terms
        self.h = nat.Handle(circuit.n, device, nat.SVB_FP64)

    def run(self, points: np.ndarray, gradients: bool = True):
        m, n_params = points.shape
        e = np.zeros(m)
        g = np.zeros((m, n_params)) if gradients else None
        for i in range(m):
            gates = self.circuit.evaluated(points[i])
            if gradients:
                e[i], g[i] = self.h.adjoint(gates, self.circuit.binding, n_params, self.terms)
            else:
                self.h.reset()
                self.h.set_circuit(gates)
                self.h.run()
                e[i] = self.h.expectation(self.terms)
        return e, g

    def close(self):
        self.h.close()


class ShardedAdjoint:
    """Energy (and adjoint gradient) of one parametrised circuit (a
    ``circuits.ParamCircuit``) for an observable (Pauli terms) at many parameter points,
    split across the ranks of `group` (torch.distributed; a single process when it is not
    initialised).

    `make_local()` builds this rank's evaluator, by default an ``AdjointPoints`` on
    `device`; its ``run(points [m, P], gradients)`` returns ``(energies [m], grads [m, P]
    or None)``."""

    def __init__(self, circuit, terms, device: int = 0, group=None, make_local: Callable | None = None):
        import torch.distributed as dist
        self.distributed = dist.is_available() and dist.is_initialized()
        self.group = group
        self.world = dist.get_world_size(group) if self.distributed else 1
        self.rank = dist.get_rank(group) if self.distributed else 0
        self.device = device
        self.n_params = len(circuit.params)
        if make_local is None:
            def make_local():
                return AdjointPoints(circuit, terms, device)
        self.local = make_local()

    def run(self, points, gradients: bool = True):
        """points: [m, P] (the same on every rank).  Returns (energies [m], grads [m, P])
        on every rank; grads is None when `gradients` is False."""
        pts = np.asarray(points, dtype=np.float64).reshape(-1, self.n_params)
        m = len(pts)
        mine = split_even(m, self.world)[self.rank]
        cols = 1 + (self.n_params if gradients else 0)
        full = np.zeros((m, cols))
        if mine:
            e, g = self.local.run(pts[mine[0]:mine[-1] + 1], gradients)
            full[mine[0]:mine[-1] + 1, 0] = e
            if gradients:
                full[mine[0]:mine[-1] + 1, 1:] = g
        full = _gather_rows(full, self.world, self.group, self.device)
        return full[:, 0].copy(), (full[:, 1:].copy() if gradients else None)

    def close(self):
        if self.local is not None and hasattr(self.local, "close"):
            self.local.close()
        self.local = None
