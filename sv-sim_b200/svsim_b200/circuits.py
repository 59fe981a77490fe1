"""Seeded synthetic workloads.

There is no public circuit suite behind these numbers: every workload is a seeded
random circuit with the shape of one measured configuration (layer recipe, qubit
count, depth, angle distribution).  The same generator feeds the CUDA path, the C
oracle and the reference CPU backends, so all of them see identical gate lists.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .gates import GATE_DTYPE, PARAM_DTYPE, PAULI_DTYPE, OP

TWO_PI = 2.0 * math.pi


def _u3_layer(rng, n, out):
    ang = rng.uniform(0.0, TWO_PI, size=(n, 3))
    for q in range(n):
        out.append((OP["U3"], (q, 0, 0, 0, 0), ang[q, 0], ang[q, 1], ang[q, 2]))


def _pack(rows) -> np.ndarray:
    arr = np.zeros(len(rows), dtype=GATE_DTYPE)
    for i, (op, qb, th, ph, la) in enumerate(rows):
        arr[i] = (op, qb, th, ph, la)
    return arr


def brickwork_circuit(n: int = 16, layers: int = 20, seed: int = 1234) -> np.ndarray:
    """U3(theta, phi, lambda) on every qubit with angles iid U[0, 2pi), then CX on a
    brickwork pairing: even layers (0,1),(2,3)..., odd layers (1,2),(3,4)...
    n=16, 20 layers: 320 U3 + 150 CX = 470 gates."""
    rng = np.random.default_rng(seed)
    rows = []
    for layer in range(layers):
        _u3_layer(rng, n, rows)
        start = layer % 2
        for a in range(start, n - 1, 2):
            rows.append((OP["CX"], (a, a + 1, 0, 0, 0), 0.0, 0.0, 0.0))
    return _pack(rows)


def random_matching_circuit(n: int = 30, depth: int = 40, seed: int = 2024) -> np.ndarray:
    """Each layer: U3 with U[0, 2pi) angles on all n qubits, then floor(n/2) CX on a
    seeded random perfect matching (control = first of the pair), so CX gates land on
    high, strided qubits.  n=30, depth 40: 1,200 U3 + 600 CX = 1,800 gates."""
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(depth):
        _u3_layer(rng, n, rows)
        perm = rng.permutation(n)
        for i in range(n // 2):
            rows.append((OP["CX"], (int(perm[2 * i]), int(perm[2 * i + 1]), 0, 0, 0),
                         0.0, 0.0, 0.0))
    return _pack(rows)


def inverse_circuit(gates: np.ndarray) -> np.ndarray:
    """The inverse gate list of a U3/CX/H/X circuit: reversed order, U3(t, p, l) ->
    U3(-t, -l, -p) (the conjugate transpose of the reference's U3 matrix), CX, H, X
    self-inverse."""
    out = np.ascontiguousarray(gates[::-1].copy())
    for g in out:
        op = int(g["op"])
        if op == OP["U3"]:
            t, p, l = float(g["theta"]), float(g["phi"]), float(g["lam"])
            g["theta"], g["phi"], g["lam"] = -t, -l, -p
        elif op not in (OP["CX"], OP["H"], OP["X"]):
            raise ValueError(f"inverse_circuit: op {op} not supported")
    return out


@dataclass
class ParamCircuit:
    """A circuit whose angles depend affinely on a parameter vector:
    angle_f(gate) = sum over its binding of coef_f * params[idx_f]."""
    n: int
    gates: np.ndarray         # GATE_DTYPE, angles evaluated at `params`
    binding: np.ndarray       # PARAM_DTYPE, one per gate
    params: np.ndarray        # float64 [P]

    def evaluated(self, params: np.ndarray) -> np.ndarray:
        """Gate records with all bound angles recomputed from `params`."""
        g = self.gates.copy()
        fields = ("theta", "phi", "lam")
        for f in range(3):
            idx = self.binding["idx"][:, f]
            m = idx >= 0
            g[fields[f]][m] = self.binding["coef"][m, f] * params[idx[m]]
        return g


def hardware_efficient_ansatz(n: int = 20, layers: int = 12, seed: int = 7) -> ParamCircuit:
    """Per layer: RY(theta) on every qubit, RZ(theta) on every qubit, CX ring i -> i+1 mod n.
    n=20, 12 layers: 720 gates, P = 480 parameters iid U[-pi, pi]."""
    rng = np.random.default_rng(seed)
    P = 2 * n * layers
    params = rng.uniform(-math.pi, math.pi, size=P)
    gates = np.zeros(3 * n * layers, dtype=GATE_DTYPE)
    binding = np.zeros(len(gates), dtype=PARAM_DTYPE)
    binding["idx"] = -1
    k = 0
    for layer in range(layers):
        for q in range(n):
            p = layer * 2 * n + q
            gates[k] = (OP["RY"], (q, 0, 0, 0, 0), params[p], 0.0, 0.0)
            binding[k]["idx"][0] = p
            binding[k]["coef"][0] = 1.0
            k += 1
        for q in range(n):
            p = layer * 2 * n + n + q
            gates[k] = (OP["RZ"], (q, 0, 0, 0, 0), 0.0, params[p], 0.0)
            binding[k]["idx"][1] = p
            binding[k]["coef"][1] = 1.0
            k += 1
        for q in range(n):
            gates[k] = (OP["CX"], (q, (q + 1) % n, 0, 0, 0), 0.0, 0.0, 0.0)
            k += 1
    return ParamCircuit(n, gates, binding, params)


def zz_x_hamiltonian(n: int = 20, x_coef: float = 0.5) -> np.ndarray:
    """H = sum_i Z_i Z_{i+1} + x_coef * sum_i X_i, periodic."""
    terms = np.zeros(2 * n, dtype=PAULI_DTYPE)
    for i in range(n):
        terms[i] = (1.0, 0, (1 << i) | (1 << ((i + 1) % n)))
        terms[n + i] = (x_coef, 1 << i, 0)
    return terms


@dataclass
class QaoaInstance:
    n: int
    edges: np.ndarray     # int32 [E, 2]
    weights: np.ndarray   # float64 [E]
    gammas: np.ndarray    # float64 [p]
    betas: np.ndarray     # float64 [p]

    def cost_table(self) -> np.ndarray:
        """C(z) = sum_e w_e [z_a != z_b] for every basis state z (MaxCut value)."""
        z = np.arange(1 << self.n, dtype=np.int64)
        c = np.zeros(1 << self.n)
        for (a, b), w in zip(self.edges, self.weights):
            c += w * (((z >> a) ^ (z >> b)) & 1)
        return c

    def circuit(self) -> np.ndarray:
        """The instance in the reference gate set: H on all, then per layer RZZ(-gamma*w)
        per edge (RZZ = CX.U1.CX, svsim_nvgpu_sin.cuh:1288-1294, applies
        e^{i theta [a != b]}) and RX(2 beta) on every qubit."""
        rows = [(OP["H"], (q, 0, 0, 0, 0), 0.0, 0.0, 0.0) for q in range(self.n)]
        for g, b in zip(self.gammas, self.betas):
            for (u, v), w in zip(self.edges, self.weights):
                rows.append((OP["RZZ"], (int(u), int(v), 0, 0, 0), -g * w, 0.0, 0.0))
            for q in range(self.n):
                rows.append((OP["RX"], (q, 0, 0, 0, 0), 2.0 * b, 0.0, 0.0))
        return _pack(rows)

    def param_circuit(self) -> ParamCircuit:
        """`circuit()` with its angles bound to params = [gamma_0..gamma_{p-1},
        beta_0..beta_{p-1}] (RZZ theta = -w_e * gamma_l, RX theta = 2 * beta_l)."""
        p = len(self.gammas)
        gates = self.circuit()
        binding = np.zeros(len(gates), dtype=PARAM_DTYPE)
        binding["idx"] = -1
        k = self.n
        for layer in range(p):
            for w in self.weights:
                binding[k]["idx"][0] = layer
                binding[k]["coef"][0] = -float(w)
                k += 1
            for _ in range(self.n):
                binding[k]["idx"][0] = p + layer
                binding[k]["coef"][0] = 2.0
                k += 1
        params = np.concatenate([self.gammas, self.betas]).astype(np.float64)
        return ParamCircuit(self.n, gates, binding, params)

    def maxcut_terms(self) -> np.ndarray:
        """C = sum_e w_e (1 - Z_a Z_b) / 2 as Pauli terms."""
        terms = np.zeros(len(self.edges) + 1, dtype=PAULI_DTYPE)
        terms[0] = (0.5 * float(np.sum(self.weights)), 0, 0)
        for k, ((a, b), w) in enumerate(zip(self.edges, self.weights)):
            terms[k + 1] = (-0.5 * float(w), 0, (1 << int(a)) | (1 << int(b)))
        return terms


def qaoa_instances(count: int = 512, n_min: int = 10, n_max: int = 22, p: int = 4,
                   edge_prob: float = 0.3, seed: int = 99) -> list[QaoaInstance]:
    """Seeded G(n, 0.3) MaxCut instances, n ~ U{n_min..n_max}, weights U[0.5, 1.5],
    gamma ~ U[0, pi], beta ~ U[0, pi/2], depth p."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(n_min, n_max + 1))
        iu, ju = np.triu_indices(n, 1)
        keep = rng.random(len(iu)) < edge_prob
        edges = np.stack([iu[keep], ju[keep]], axis=1).astype(np.int32)
        if len(edges) == 0:
            edges = np.array([[0, 1]], dtype=np.int32)
        weights = rng.uniform(0.5, 1.5, size=len(edges))
        gammas = rng.uniform(0.0, math.pi, size=p)
        betas = rng.uniform(0.0, math.pi / 2, size=p)
        out.append(QaoaInstance(n, edges, weights, gammas, betas))
    return out
