"""Density-matrix simulation with noise (the reference's svsim_qsharp_noise variant).

rho of n qubits lives on the GPU as an FP64 vector of 2n qubits, rho[i][j] at index
i + 2^n j.  A circuit of reference gates runs as rho -> U rho U^dagger; an optional
one-qubit noise channel (Kraus operators) follows every gate on each qubit it touches.
The superoperator blocks run on the pair engine (FP64 tensor cores) for n >= 6 and as
per-gate sweeps below.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat
from .gates import GATE_DTYPE, OP

SUPEROP_DTYPE = np.dtype([("op", np.uint32), ("reserved", np.uint32), ("m", np.float64, (32,))])


def depolarizing(p: float):
    """rho -> (1 - p) rho + p/3 (X rho X + Y rho Y + Z rho Z)."""
    i = np.eye(2)
    x = np.array([[0, 1], [1, 0]])
    y = np.array([[0, -1j], [1j, 0]])
    z = np.diag([1, -1])
    return [np.sqrt(1 - p) * i, np.sqrt(p / 3) * x, np.sqrt(p / 3) * y, np.sqrt(p / 3) * z]


def pauli_channel(p_i: float, p_x: float, p_y: float, p_z: float):
    """rho -> p_i rho + p_x X rho X + p_y Y rho Y + p_z Z rho Z."""
    i = np.eye(2)
    x = np.array([[0, 1], [1, 0]])
    y = np.array([[0, -1j], [1j, 0]])
    z = np.diag([1, -1])
    return [np.sqrt(p_i) * i, np.sqrt(p_x) * x, np.sqrt(p_y) * y, np.sqrt(p_z) * z]


def superoperator(kraus, unitary=None):
    """4x4 superoperator of rho -> sum_k K_k (U rho U^dagger) K_k^dagger in the reference's
    table order (svsim_qsharp_noise/noise_gate_*.cuh): entry [r, c] with r = 2 i + j for
    rho[i][j], so that rho'_r = sum_c S[r, c] rho_c."""
    u = np.eye(2) if unitary is None else np.asarray(unitary, dtype=np.complex128)
    s = np.zeros((4, 4), dtype=np.complex128)
    for k in kraus:
        m = np.asarray(k, dtype=np.complex128) @ u
        s += np.kron(m, m.conj())
    return s


def amplitude_damping(gamma: float):
    return [np.array([[1, 0], [0, np.sqrt(1 - gamma)]]), np.array([[0, np.sqrt(gamma)], [0, 0]])]


def phase_damping(lam: float):
    return [np.array([[1, 0], [0, np.sqrt(1 - lam)]]), np.array([[0, 0], [0, np.sqrt(lam)]])]


def bit_flip(p: float):
    return [np.sqrt(1 - p) * np.eye(2), np.sqrt(p) * np.array([[0, 1], [1, 0]])]


class DensityMatrix:
    def __init__(self, n_qubits: int, device: int = 0):
        h = ctypes.c_void_p()
        nat.check(nat.lib().svb_dm_create(n_qubits, device, ctypes.byref(h)))
        self.handle = nat.Handle.__new__(nat.Handle)    # shares Handle's run/state/close
        self.handle.ptr = h
        self.handle.n = 2 * n_qubits
        self.handle.precision = nat.SVB_FP64
        self.n = n_qubits

    def set_circuit(self, gates, kraus=None, superops=None):
        """`kraus`: one-qubit channel applied after every gate to each qubit it touches.
        `superops`: {op name or enum value: 4x4 complex superoperator in the reference's
        table order (see ``superoperator``)} for one-qubit ops; such a gate is applied as
        its superoperator alone, noise included, like the reference's noisy gates."""
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        ks = [np.asarray(k, dtype=np.complex128).reshape(2, 2) for k in (kraus or [])]
        flat = np.zeros(max(1, 8 * len(ks)))
        for i, k in enumerate(ks):
            flat[8 * i:8 * i + 8] = np.stack([k.real, k.imag], axis=-1).reshape(-1)
        so = np.zeros(len(superops or {}), dtype=SUPEROP_DTYPE)
        for i, (op, m) in enumerate((superops or {}).items()):
            m = np.asarray(m, dtype=np.complex128).reshape(4, 4)
            so[i]["op"] = OP[op] if isinstance(op, str) else int(op)
            so[i]["m"] = np.stack([m.real, m.imag], axis=-1).reshape(-1)
        nat.check(nat.lib().svb_dm_set_circuit_superops(self.handle.ptr, g.ctypes.data, len(g), nat.dptr(flat),
                                                        len(ks), so.ctypes.data if len(so) else None, len(so)))
        return self

    def run(self):
        self.handle.run()
        self.handle.sync()

    def reset(self):
        self.handle.reset()

    def probabilities(self) -> np.ndarray:
        out = np.zeros(1 << self.n)
        nat.check(nat.lib().svb_dm_probabilities(self.handle.ptr, nat.dptr(out)))
        return out

    def rho(self) -> np.ndarray:
        """The full density matrix on the host (small n)."""
        re, im = self.handle.get_state()
        d = 1 << self.n
        return (re + 1j * im).reshape(d, d).T           # rho[i][j] at i + d j

    def measure(self, uniforms) -> np.ndarray:
        """Samples with the reference's rule (first j with S_j <= r < S_{j+1}, else 0) on
        the probabilities."""
        cdf = np.cumsum(self.probabilities())
        u = np.asarray(uniforms, dtype=np.float64)
        j = np.searchsorted(cdf, u, side="right")
        return np.where(j < len(cdf), j, 0).astype(np.uint64)

    def plan_info(self):
        return self.handle.plan_info()

    def close(self):
        self.handle.close()
