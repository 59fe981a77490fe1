"""Gate records and the reference's gate vocabulary.

The op numbering is the reference's ``enum OP`` (svsim/src/svsim_nvgpu_sin.cuh:42-48),
and a gate record carries the same fields as ``class Gate`` (:99-188): the op, five
qubit slots and the three angles theta, phi, lambda.  Which angle an op reads follows
the ``*_OP`` wrappers (:1459-1647): U3 reads all three, U2 reads (phi, lambda), U1, CRX,
CRY, CRZ and CU1 read lambda, RZ reads phi, and RX, RY, R, RXX, RZZ, RYY read theta.
The static factories below keep the argument order of ``Simulation::U3`` ... ``RYY``
(:397-584).
"""
from __future__ import annotations

import numpy as np

OP_NAMES = (
    "U3", "U2", "U1", "CX", "ID", "X", "Y", "Z", "H", "S",
    "SDG", "T", "TDG", "RX", "RY", "RZ", "CZ", "CY", "SWAP", "CH",
    "CCX", "CSWAP", "CRX", "CRY", "CRZ", "CU1", "CU3", "RXX", "RZZ", "RCCX",
    "RC3X", "C3X", "C3SQRTX", "C4X", "R", "SRN", "W", "RYY",
)
OP = {name: i for i, name in enumerate(OP_NAMES)}
globals().update({f"OP_{k}": v for k, v in OP.items()})

# number of qubit slots each op uses
N_QUBITS = {
    **{k: 1 for k in ("U3", "U2", "U1", "ID", "X", "Y", "Z", "H", "S", "SDG", "T", "TDG",
                      "RX", "RY", "RZ", "R", "SRN", "W")},
    **{k: 2 for k in ("CX", "CZ", "CY", "SWAP", "CH", "CRX", "CRY", "CRZ", "CU1", "CU3",
                      "RXX", "RZZ", "RYY")},
    **{k: 3 for k in ("CCX", "CSWAP", "RCCX")},
    **{k: 4 for k in ("RC3X", "C3X", "C3SQRTX")},
    "C4X": 5,
}

# byte layout of svb_gate (include/svsim_b200.h): 48 bytes
GATE_DTYPE = np.dtype([("op", "<u4"), ("qb", "<u4", (5,)),
                       ("theta", "<f8"), ("phi", "<f8"), ("lam", "<f8")])
assert GATE_DTYPE.itemsize == 48

# parameter binding of a gate for the adjoint: per angle field (theta, phi, lambda)
# the index of the circuit parameter it depends on (-1: none) and d(angle)/d(param).
PARAM_DTYPE = np.dtype([("idx", "<i4", (3,)), ("pad", "<i4"), ("coef", "<f8", (3,))])
assert PARAM_DTYPE.itemsize == 40

# Pauli term of an observable: coef * prod_q sigma_q, sigma encoded by two masks
PAULI_DTYPE = np.dtype([("coef", "<f8"), ("x_mask", "<u8"), ("z_mask", "<u8")])


class Gate:
    """One gate record, with the constructor of the reference's ``Gate`` (:102-107)."""

    __slots__ = ("op", "qb", "theta", "phi", "lam")

    def __init__(self, op, qb0=0, qb1=0, qb2=0, qb3=0, qb4=0, theta=0.0, phi=0.0, lam=0.0):
        self.op = int(op)
        self.qb = (int(qb0), int(qb1), int(qb2), int(qb3), int(qb4))
        self.theta, self.phi, self.lam = float(theta), float(phi), float(lam)

    @property
    def name(self):
        return OP_NAMES[self.op]

    def qubits(self):
        return self.qb[: N_QUBITS[self.name]]

    def __repr__(self):
        # same text as Gate::dump (:167-173)
        return (f"{self.name}({self.qb[0]},{self.qb[1]},{self.qb[2]},{self.qb[3]},"
                f"{self.qb[4]},{self.theta:g},{self.phi:g},{self.lam:g});")


def to_array(gates) -> np.ndarray:
    """Pack Gate objects (or an existing record array) into svb_gate records."""
    if isinstance(gates, np.ndarray) and gates.dtype == GATE_DTYPE:
        return np.ascontiguousarray(gates)
    arr = np.zeros(len(gates), dtype=GATE_DTYPE)
    for i, g in enumerate(gates):
        arr[i] = (g.op, g.qb, g.theta, g.phi, g.lam)
    return arr


def from_array(arr: np.ndarray):
    return [Gate(int(r["op"]), *[int(x) for x in r["qb"]], float(r["theta"]),
                 float(r["phi"]), float(r["lam"])) for r in arr]


# ---- static factories, argument order of Simulation::U3 ... RYY (:397-584) ----
def U3(theta, phi, lam, m): return Gate(OP_U3, m, 0, 0, 0, 0, theta, phi, lam)
def U2(phi, lam, m): return Gate(OP_U2, m, 0, 0, 0, 0, 0.0, phi, lam)
def U1(lam, m): return Gate(OP_U1, m, 0, 0, 0, 0, 0.0, 0.0, lam)
def CX(m, n): return Gate(OP_CX, m, n)
def ID(m): return Gate(OP_ID, m)
def X(m): return Gate(OP_X, m)
def Y(m): return Gate(OP_Y, m)
def Z(m): return Gate(OP_Z, m)
def H(m): return Gate(OP_H, m)
def S(m): return Gate(OP_S, m)
def SDG(m): return Gate(OP_SDG, m)
def T(m): return Gate(OP_T, m)
def TDG(m): return Gate(OP_TDG, m)
def RX(theta, m): return Gate(OP_RX, m, 0, 0, 0, 0, theta, 0.0, 0.0)
def RY(theta, m): return Gate(OP_RY, m, 0, 0, 0, 0, theta, 0.0, 0.0)
def RZ(phi, m): return Gate(OP_RZ, m, 0, 0, 0, 0, 0.0, phi, 0.0)
def CZ(m, n): return Gate(OP_CZ, m, n)
def CY(m, n): return Gate(OP_CY, m, n)
def SWAP(m, n): return Gate(OP_SWAP, m, n)
def CH(m, n): return Gate(OP_CH, m, n)
def CCX(l, m, n): return Gate(OP_CCX, l, m, n)
def CSWAP(l, m, n): return Gate(OP_CSWAP, l, m, n)
def CRX(lam, m, n): return Gate(OP_CRX, m, n, 0, 0, 0, 0.0, 0.0, lam)
def CRY(lam, m, n): return Gate(OP_CRY, m, n, 0, 0, 0, 0.0, 0.0, lam)
def CRZ(lam, m, n): return Gate(OP_CRZ, m, n, 0, 0, 0, 0.0, 0.0, lam)
def CU1(lam, m, n): return Gate(OP_CU1, m, n, 0, 0, 0, 0.0, 0.0, lam)
def CU3(theta, phi, lam, m, n): return Gate(OP_CU3, m, n, 0, 0, 0, theta, phi, lam)
def RXX(theta, m, n): return Gate(OP_RXX, m, n, 0, 0, 0, theta, 0.0, 0.0)
def RZZ(theta, m, n): return Gate(OP_RZZ, m, n, 0, 0, 0, theta, 0.0, 0.0)
def RCCX(l, m, n): return Gate(OP_RCCX, l, m, n)
def RC3X(l, m, n, o): return Gate(OP_RC3X, l, m, n, o)
def C3X(l, m, n, o): return Gate(OP_C3X, l, m, n, o)
def C3SQRTX(l, m, n, o): return Gate(OP_C3SQRTX, l, m, n, o)
def C4X(l, m, n, o, p): return Gate(OP_C4X, l, m, n, o, p)
def R(theta, m): return Gate(OP_R, m, 0, 0, 0, 0, theta, 0.0, 0.0)
def SRN(m): return Gate(OP_SRN, m)
def W(m): return Gate(OP_W, m)
def RYY(theta, m, n): return Gate(OP_RYY, m, n, 0, 0, 0, theta, 0.0, 0.0)

FACTORIES = {name: globals()[name] for name in OP_NAMES}
