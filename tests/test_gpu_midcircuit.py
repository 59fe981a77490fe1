"""Immediate-mode operations of the Q#/QIR variant: masked multi-controlled gates and
mid-circuit Pauli measurement with collapse, against a numpy restatement of the
variant's kernels (ControlledX ... with OP_HEAD_MASK, Measure_GATE) on the oracle's
state."""
import numpy as np
import pytest

from svsim_b200 import circuits

pytestmark = pytest.mark.gpu

S2I = 1 / np.sqrt(2)
H = np.array([[S2I, S2I], [S2I, -S2I]])
S = np.diag([1, 1j])
SDG = np.diag([1, -1j])


def apply_1q(psi, q, u, controls=()):
    """u on qubit q where every control bit is 1 (the OP_HEAD_MASK rule)."""
    out = psi.copy()
    idx = np.arange(len(psi))
    sel = ((idx >> q) & 1) == 0
    for c in controls:
        sel &= ((idx >> c) & 1) == 1
    i0 = idx[sel]
    i1 = i0 | (1 << q)
    a0, a1 = psi[i0], psi[i1]
    out[i0] = u[0, 0] * a0 + u[0, 1] * a1
    out[i1] = u[1, 0] * a0 + u[1, 1] * a1
    return out


def measure_ref(psi, q, pauli, r):
    """Measure_GATE: basis change, P(1), outcome = r < P(1), collapse, basis back."""
    if pauli == 1:
        psi = apply_1q(psi, q, H)
    if pauli == 2:
        psi = apply_1q(apply_1q(psi, q, SDG), q, H)
    idx = np.arange(len(psi))
    one = ((idx >> q) & 1) == 1
    p1 = float(np.sum(np.abs(psi[one]) ** 2))
    outcome = 1 if r < p1 else 0
    keep = one if outcome else ~one
    psi = np.where(keep, psi / np.sqrt(p1 if outcome else 1 - p1), 0)
    if pauli == 1:
        psi = apply_1q(psi, q, H)
    if pauli == 2:
        psi = apply_1q(apply_1q(psi, q, H), q, S)
    return psi, outcome, p1


def random_state_handle(n, precision=0, seed=1):
    from svsim_b200 import _native as nat
    g = circuits.random_matching_circuit(n, 4, seed=seed)
    h = nat.Handle(n, 0, precision)
    h.set_circuit(g)
    h.run()
    h.sync()
    re, im = h.get_state()
    return h, re + 1j * im


def random_unitary(rng):
    z = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


@pytest.mark.parametrize("controls", [(), (3,), (0, 7), (2, 9, 11, 12)])
def test_masked_controlled_gate(controls):
    rng = np.random.default_rng(len(controls))
    n = 13
    h, psi = random_state_handle(n)
    u = random_unitary(rng)
    target = 5
    h.apply_controlled(target, controls, u)
    h.sync()
    re, im = h.get_state()
    ref = apply_1q(psi, target, u, controls)
    assert np.max(np.abs((re + 1j * im) - ref)) <= 1e-14


@pytest.mark.parametrize("pauli", [0, 1, 2])
def test_mid_circuit_measurement_collapses(pauli):
    n = 14
    for q, r in [(0, 0.3), (6, 0.71), (13, 0.05)]:
        h, psi = random_state_handle(n, seed=q + 3 * pauli)
        outcome, p1 = h.measure_qubit(q, r, pauli)
        ref, ro, rp1 = measure_ref(psi, q, pauli, r)
        assert outcome == ro and abs(p1 - rp1) <= 1e-13
        re, im = h.get_state()
        assert np.max(np.abs((re + 1j * im) - ref)) <= 1e-13
        assert abs(h.norm2() - 1.0) <= 1e-12


def test_measurement_then_circuit_and_fp32():
    """A measured qubit in Z reads the same outcome again; an FP32 state follows FP64."""
    from svsim_b200 import _native as nat
    n = 12
    h, _ = random_state_handle(n)
    o1, p1 = h.measure_qubit(4, 0.5, 0)
    o2, p2 = h.measure_qubit(4, 0.99, 0)
    assert o1 == o2 and abs(p2 - float(o1)) <= 1e-12
    h32, _ = random_state_handle(n, precision=nat.SVB_FP32)
    h64, _ = random_state_handle(n, precision=nat.SVB_FP64)
    a = h32.measure_qubit(3, 0.4, 1)
    b = h64.measure_qubit(3, 0.4, 1)
    assert a[0] == b[0] and abs(a[1] - b[1]) <= 1e-5
    f, d = h64.compare(h32)
    assert 1 - f <= 1e-6


def test_invalid_arguments():
    from svsim_b200 import _native as nat
    h, _ = random_state_handle(8)
    with pytest.raises(nat.SvbError):
        h.apply_controlled(3, (3,), np.eye(2))
    with pytest.raises(nat.SvbError):
        h.apply_controlled(9, (), np.eye(2))
    with pytest.raises(nat.SvbError):
        h.measure_qubit(8, 0.5, 0)
    with pytest.raises(nat.SvbError):
        h.measure_qubit(1, 0.5, 3)
