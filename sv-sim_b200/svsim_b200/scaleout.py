"""One circuit on several GPUs: the state split by its high qubits, qubit-swap exchanges.

Replaces the multi-GPU variants of the reference (svsim/src/svsim_nvgpu_mpi.cuh and
svsim_nvgpu_omp.cuh).  As there, R = 2^r ranks each hold 2^(n-r) amplitudes and the top r
index bits name the rank (svsim_nvgpu_mpi.cuh:244-246: gpu_scale, lg2_m_gpu).  The
reference applies every gate to remote amplitudes element by element through NVSHMEM
gets and puts (:761-810).  Here:

* the circuit is cut into segments whose gates touch only rank-local qubits; each segment
  runs on the rank's own chunk with the single-GPU engines, its qubits renamed to the
  physical bit positions they currently occupy;
* between segments one exchange step swaps r local qubits with the r rank bits: SWAP
  gates first move the outgoing qubits to the top r local positions, then one
  all-to-all (NCCL over NVLink) transposes those positions with the rank bits.  The
  qubits that go out are the local ones whose next use is furthest away (Belady);
* after the circuit the logical qubit order is restored, so the gathered state and the
  samples follow the reference's index order.

The physical layout is a permutation pi: logical qubit q sits at bit position pi[q];
positions 0..m-1 (m = n - r) are local, m..n-1 are the rank bits.  SWAP is a permutation
of amplitudes and a gate on renamed qubits does the same arithmetic on the same values,
so the result is the single-GPU result exactly.

The compute side of a rank is a chunk backend (`GpuChunk`: an svb handle on the rank's
GPU); the exchange is `torch.distributed.all_to_all_single` over the process group
(NCCL for CUDA tensors).  No kernel waits on another rank: the only cross-rank step is
the collective, taken by every rank in the same order.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import gates as G

INF = 1 << 30


def gate_qubits(rec) -> List[int]:
    name = G.OP_NAMES[int(rec["op"])]
    return [int(x) for x in rec["qb"][:G.N_QUBITS[name]]]


class Plan:
    """Steps for one rank layout: ("run", gate array on physical positions) and
    ("exchange", None).  `final_pi` is the layout after the last step."""

    def __init__(self):
        self.steps: List[Tuple[str, Optional[np.ndarray]]] = []
        self.final_pi: List[int] = []
        self.n_exchanges = 0


def plan_scaleout(gates: np.ndarray, n: int, r: int, restore: bool = True,
                  pi: Optional[Sequence[int]] = None) -> Plan:
    """Cuts `gates` (logical qubits) into local segments and exchange steps for 2^r ranks."""
    if r < 0 or r > n - 2:
        raise ValueError("scale-out needs 0 <= r <= n - 2 rank bits")
    m = n - r
    pi = list(range(n)) if pi is None else list(pi)
    where = [0] * n                       # physical position -> logical qubit
    for q, p in enumerate(pi):
        where[p] = q
    qs_of = [gate_qubits(g) for g in gates]
    for qs in qs_of:
        if len(set(qs)) != len(qs) or any(q < 0 or q >= n for q in qs):
            raise ValueError("gate qubits must be distinct and < n")
        if len(qs) > m:
            raise ValueError(f"a gate on {len(qs)} qubits needs at least that many local qubits")
    plan = Plan()
    cur: List = []

    def emit_run():
        if cur:
            plan.steps.append(("run", np.array(cur, dtype=G.GATE_DTYPE)))
            cur.clear()

    def swap_phys(a: int, b: int):
        # SWAP of physical positions a and b (both local), and the layout update
        cur.append(G.to_array([G.SWAP(a, b)])[0])
        qa, qb = where[a], where[b]
        where[a], where[b] = qb, qa
        pi[qa], pi[qb] = b, a

    def exchange(outgoing: List[int]):
        # outgoing: r logical qubits, all local; they go to the rank bits in this order
        for j, q in enumerate(outgoing):
            target = m - r + j
            if pi[q] != target:
                swap_phys(pi[q], target)
        emit_run()
        plan.steps.append(("exchange", None))
        plan.n_exchanges += 1
        for j in range(r):
            a, b = m - r + j, m + j            # top local position j <-> rank bit j
            qa, qb = where[a], where[b]
            where[a], where[b] = qb, qa
            pi[qa], pi[qb] = b, a

    def next_use(i: int) -> List[int]:
        nu = [INF] * n
        for k in range(len(qs_of) - 1, i - 1, -1):
            for q in qs_of[k]:
                nu[q] = k
        return nu

    for i, (g, qs) in enumerate(zip(gates, qs_of)):
        if r > 0 and any(pi[q] >= m for q in qs):
            nu = next_use(i)
            keep = set(qs)
            local = [q for q in range(n) if pi[q] < m and q not in keep]
            if len(local) < r:
                raise ValueError(f"a {len(qs)}-qubit gate leaves fewer than {r} other local qubits")
            local.sort(key=lambda q: -nu[q])           # furthest next use goes out
            exchange(local[:r])
        rec = g.copy()
        for k, q in enumerate(qs):
            rec["qb"][k] = pi[q]
        cur.append(rec)

    if restore and r > 0 and pi != list(range(n)):
        high = list(range(m, n))              # the logical qubits that belong on the rank bits
        if not all(pi[q] == q for q in high):
            if any(pi[q] >= m for q in high):
                # some of them are global on the wrong bit: bring every global qubit in
                out = [q for q in range(m) if pi[q] < m][:r]
                if len(out) < r:
                    raise ValueError("restoring the qubit order needs n >= 3 r")
                exchange(out)
            exchange(high)                    # high[j] -> rank bit m + j = high[j]
        for p in range(m):                    # then the local positions into order
            if pi[p] != p:
                swap_phys(pi[p], p)
    emit_run()
    plan.final_pi = list(pi)
    return plan


class GpuChunk:
    """The rank's 2^(n-r) amplitudes in an svb handle on its GPU, with a zero-copy torch
    view of the interleaved (re, im) array for the exchange."""

    def __init__(self, m: int, device: int, precision: int):
        import torch
        from . import _native as nat
        self.h = nat.Handle(m, device, precision)
        self.m = m
        self.device = device
        ptr, prec = self.h.device_ptr()
        itemsize = 8 if prec == nat.SVB_FP64 else 4

        class _View:
            __cuda_array_interface__ = {"shape": (2 << m,), "typestr": "<f8" if itemsize == 8 else "<f4",
                                        "data": (ptr, False), "version": 3, "strides": None}
        self.view = torch.as_tensor(_View(), device=f"cuda:{device}")
        self.scratch = torch.empty_like(self.view)

    def run(self, gates: np.ndarray):
        self.h.set_circuit(gates)
        self.h.run()

    def sync(self):
        import torch
        torch.cuda.synchronize(self.device)
        self.h.sync()

    def reset(self, rank: int):
        """|0..0> overall: amplitude 1 on rank 0's first entry, zero elsewhere."""
        import torch
        self.h.reset()
        self.h.sync()
        if rank != 0:
            self.view.zero_()
            torch.cuda.synchronize(self.device)

    def state(self) -> Tuple[np.ndarray, np.ndarray]:
        return self.h.get_state()

    def measure(self, uniforms: np.ndarray) -> Tuple[np.ndarray, float]:
        return self.h.measure(uniforms)

    def norm2(self) -> float:
        return self.h.norm2()

    def close(self):
        self.h.close()


class ScaleOutSimulation:
    """One circuit over the ranks of a torch.distributed process group (2^r ranks)."""

    def __init__(self, n_qubits: int, chunk=None, group=None, device: Optional[int] = None,
                 precision: Optional[int] = None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        r = self.world.bit_length() - 1
        if (1 << r) != self.world:
            raise ValueError("the number of ranks must be a power of two")
        self.n, self.r, self.m = n_qubits, r, n_qubits - r
        if chunk is None:
            from . import _native as nat
            chunk = GpuChunk(self.m, 0 if device is None else device,
                             nat.SVB_FP64 if precision is None else precision)
        self.chunk = chunk
        # small collectives (probabilities, samples, gathers) on the backend's device
        self.cdev = f"cuda:{chunk.device}" if dist.get_backend(group) == "nccl" else "cpu"
        self.pi = list(range(n_qubits))
        self.chunk.reset(self.rank)
        self.last_plan: Optional[Plan] = None

    def reset(self):
        self.pi = list(range(self.n))
        self.chunk.reset(self.rank)

    def _exchange(self):
        """Transposes the top r local positions with the r rank bits: block j of every
        rank's chunk (top local bits = j) goes to rank j, arriving as block = sender."""
        c = self.chunk
        c.sync()
        self.dist.all_to_all_single(c.scratch, c.view, group=self.group)
        c.view.copy_(c.scratch)
        c.sync()

    def run(self, gates: np.ndarray, restore: bool = True) -> Plan:
        plan = plan_scaleout(np.ascontiguousarray(gates, dtype=G.GATE_DTYPE), self.n, self.r,
                             restore=restore, pi=self.pi)
        for kind, g in plan.steps:
            if kind == "run":
                self.chunk.run(g)
            else:
                self._exchange()
        self.chunk.sync()
        self.pi = plan.final_pi
        self.last_plan = plan
        return plan

    def gather_state(self) -> Optional[Tuple[np.ndarray, np.ndarray]]:
        """The full state in logical order on rank 0 (None elsewhere); for checks and
        small states (every rank takes part)."""
        import torch
        re, im = self.chunk.state()
        parts = torch.from_numpy(np.stack([re, im])).to(self.cdev)
        got = [torch.empty_like(parts) for _ in range(self.world)]
        self.dist.all_gather(got, parts, group=self.group)
        if self.rank != 0:
            return None
        full = torch.cat([p.cpu() for p in got], dim=1).numpy()
        re_p, im_p = full[0], full[1]
        if self.pi == list(range(self.n)):
            return re_p.copy(), im_p.copy()
        # physical index -> logical index
        idx = np.arange(1 << self.n, dtype=np.int64)
        logical = np.zeros_like(idx)
        for q, p in enumerate(self.pi):
            logical |= ((idx >> p) & 1) << q
        re_l = np.empty_like(re_p)
        im_l = np.empty_like(im_p)
        re_l[logical] = re_p
        im_l[logical] = im_p
        return re_l, im_l

    def measure(self, uniforms: np.ndarray) -> np.ndarray:
        """Samples with the reference's rule over the whole state (index order, default 0
        when r is past the total), the layout restored; every rank returns them."""
        import torch
        if self.pi != list(range(self.n)):
            raise RuntimeError("measure needs the logical qubit order (run with restore=True)")
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        p_local = torch.tensor([self.chunk.norm2()], dtype=torch.float64, device=self.cdev)
        allp = [torch.zeros(1, dtype=torch.float64, device=self.cdev) for _ in range(self.world)]
        self.dist.all_gather(allp, p_local, group=self.group)
        p = np.array([float(t.item()) for t in allp])
        start = np.concatenate([[0.0], np.cumsum(p)[:-1]])
        mine = (u >= start[self.rank]) & (u < start[self.rank] + p[self.rank])
        out = np.zeros(len(u), dtype=np.int64)
        if mine.any():
            s, _ = self.chunk.measure(u[mine] - start[self.rank])
            out[mine] = s.astype(np.int64) + (self.rank << self.m)
        t = torch.from_numpy(out).to(self.cdev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy().astype(np.uint64)

    def close(self):
        self.chunk.close()
