"""Density matrices pinned to the reference's noise variant (svsim_qsharp_noise/), through
tests/golden/noise.npz (made from the reference files by make_golden_noise.py):

  * its superoperator tables noise_gate_{DP,AD,BCSZ}_{0.99,0.98}.cuh, given as per-op
    superoperators, are applied by the GPU exactly as its C2_GATE applies them
    (svsim_nvgpu_sin.cuh:1727-1800, restated here on the 2^(2n) vector);
  * the depolarizing tables of X, Y and Z are the gate followed by a Pauli channel, and
    density.superoperator(pauli_channel(...), gate) rebuilds them to rounding: the
    Kraus -> superoperator construction and its index order are the reference's;
  * its 32 unit tests (unit_test_nvgpu_sin.cu), mapped onto the reference gate set, give
    its expected density matrices within its ERROR_BAR."""
import math

import numpy as np
import pytest

from conftest import load_golden
from svsim_b200 import density as D, gates as G

GPU = pytest.mark.gpu

PAULI = {"I": np.eye(2), "X": np.array([[0, 1], [1, 0]]), "Y": np.array([[0, -1j], [1j, 0]]),
         "Z": np.diag([1.0, -1.0])}


@pytest.fixture(scope="module")
def noise():
    return load_golden("noise.npz")


def c2_gate(vec, n, q, e):
    """C2_GATE of the noise variant on the (row q, column q) pair of a 2^(2n) vector:
    pos0..pos3 = base, base + 2^(q+n), base + 2^q, base + both; out[r] = sum_c e[r, c] in[c]."""
    v = vec.copy()
    d1, d0 = 1 << (q + n), 1 << q
    for base in range(1 << (2 * n)):
        if base & d0 or base & d1:
            continue
        pos = [base, base + d1, base + d0, base + d0 + d1]
        x = v[pos]
        v[pos] = e @ x
    return v


def test_depolarizing_tables_are_gate_then_pauli_channel(noise):
    """CPU: DP tables of X, Y, Z = superoperator(pauli_channel(p), gate) with
    p = (p_I, p_X, p_Y, p_Z) solved from the table; our builder reproduces every entry."""
    names = list(noise["table_names"])
    gates = list(noise["table_gates"])
    for tname in ("DP_0.99", "DP_0.98"):
        t = noise["tables"][names.index(tname)]
        for g in "XYZ":
            table = t[gates.index(g)].reshape(4, 4)
            basis = [D.superoperator([PAULI[p]], PAULI[g]) for p in "IXYZ"]
            A = np.array([b.reshape(-1) for b in basis]).T
            p = np.linalg.lstsq(A, table.reshape(-1), rcond=None)[0].real
            assert np.all(p >= 0) and abs(p.sum() - 1) <= 1e-12
            rebuilt = D.superoperator(D.pauli_channel(*p), PAULI[g])
            assert np.max(np.abs(rebuilt - table)) <= 1e-15, (tname, g)


@GPU
@pytest.mark.parametrize("tname", ["DP_0.99", "DP_0.98", "AD_0.99", "AD_0.98", "BCSZ_0.99", "BCSZ_0.98"])
def test_noise_tables_applied_like_c2_gate(noise, tname):
    names = list(noise["table_names"])
    tables = noise["tables"][names.index(tname)]
    sup = {g: tables[i].reshape(4, 4) for i, g in enumerate(noise["table_gates"])}
    n = 4
    rng = np.random.default_rng(len(tname))
    gl = []
    for _ in range(24):
        g = "XYZH"[rng.integers(4)]
        gl.append(getattr(G, g)(int(rng.integers(n))))
    gl.insert(5, G.CX(0, 2))                         # noiseless gates stay U rho U^dagger
    gl.insert(11, G.RY(0.7, 3))
    dm = D.DensityMatrix(n)
    dm.set_circuit(G.to_array(gl), superops=sup)
    dm.run()
    re, im = dm.handle.get_state()
    got = re + 1j * im
    # the restatement: rho as the reference's vector, C2_GATE for the tabled gates
    vec = np.zeros(1 << (2 * n), dtype=complex)
    vec[0] = 1.0
    for g in gl:
        name = g.name
        if name in sup:
            vec = c2_gate(vec, n, g.qb[0], sup[name])
        else:
            rho = vec.reshape(1 << n, 1 << n).T
            full = ry_or_cx(n, g)
            rho = full @ rho @ full.conj().T
            vec = rho.T.reshape(-1)
    assert np.max(np.abs(got - vec)) <= 1e-14


def ry_or_cx(n, g):
    d = 1 << n
    m = np.zeros((d, d), dtype=complex)
    if g.name == "CX":
        c, t = g.qb[0], g.qb[1]
        for k in range(d):
            m[k ^ (1 << t) if (k >> c) & 1 else k, k] = 1.0
        return m
    th = g.theta
    r = np.array([[math.cos(th / 2), -math.sin(th / 2)], [math.sin(th / 2), math.cos(th / 2)]])
    out = np.eye(1)
    for j in reversed(range(n)):
        out = np.kron(out, r if j == g.qb[0] else np.eye(2))
    return out


def map_qsharp_op(name, args):
    """The noise variant's operations (Q# intrinsics) as reference gates.  Q#'s
    R(P, t) = exp(-i t P / 2), Exp(P, t) = exp(i t P); global phases drop out of rho, and
    a controlled global phase is a phase on the control.  Controlled ops take
    (args..., target, control_mask)."""
    if name.startswith("Controlled"):
        base = name[len("Controlled"):]
        mask = int(args[-1])
        ctrl = [q for q in range(64) if (mask >> q) & 1]
        assert len(ctrl) == 1
        c, t = ctrl[0], int(args[-2])
        th = args[0] if len(args) == 3 else None
        table = {"X": lambda: G.CX(c, t), "Y": lambda: G.CY(c, t), "Z": lambda: G.CZ(c, t),
                 "H": lambda: G.CH(c, t), "S": lambda: G.CU1(math.pi / 2, c, t),
                 "T": lambda: G.CU1(math.pi / 4, c, t), "AdjointS": lambda: G.CU1(-math.pi / 2, c, t),
                 "AdjointT": lambda: G.CU1(-math.pi / 4, c, t), "RI": lambda: G.U1(-th / 2, c),
                 "RX": lambda: G.CRX(th, c, t), "RY": lambda: G.CRY(th, c, t), "RZ": lambda: G.CRZ(th, c, t),
                 "EI": lambda: G.U1(th, c), "EX": lambda: G.CRX(-2 * th, c, t),
                 "EY": lambda: G.CRY(-2 * th, c, t), "EZ": lambda: G.CRZ(-2 * th, c, t)}
        return [table[base]()]
    q = int(args[-1])
    th = args[0] if len(args) == 2 else None
    table = {"X": lambda: G.X(q), "Y": lambda: G.Y(q), "Z": lambda: G.Z(q), "H": lambda: G.H(q),
             "S": lambda: G.S(q), "T": lambda: G.T(q), "AdjointS": lambda: G.SDG(q), "AdjointT": lambda: G.TDG(q),
             "RI": lambda: None, "EI": lambda: None, "RX": lambda: G.RX(th, q), "RY": lambda: G.RY(th, q),
             "RZ": lambda: G.RZ(th, q), "EX": lambda: G.RX(-2 * th, q), "EY": lambda: G.RY(-2 * th, q),
             "EZ": lambda: G.RZ(-2 * th, q)}
    g = table[name]()
    return [] if g is None else [g]


@GPU
def test_noise_variant_unit_tests(noise):
    failed = []
    for name, n, gl, er, ei in kat_circuits(noise):
        dm = D.DensityMatrix(n)
        dm.set_circuit(G.to_array(gl) if gl else np.zeros(0, dtype=G.GATE_DTYPE))
        dm.run()
        re, im = dm.handle.get_state()
        if np.max(np.abs(re - er)) > 1e-3 or np.max(np.abs(im - ei)) > 1e-3:
            failed.append(name)
        dm.close()
    assert not failed, failed


def kat_circuits(noise):
    pos = 0
    for k, name in enumerate(noise["kat_names"]):
        n = int(noise["kat_n"][k])
        dim = 1 << (2 * n)
        gl = []
        for op, args, kat in zip(noise["op_names"], noise["op_args"], noise["op_kat"]):
            if kat == k:
                gl += map_qsharp_op(str(op), [a for a in args if not np.isnan(a)])
        yield str(name), n, gl, noise["kat_re"][pos:pos + dim], noise["kat_im"][pos:pos + dim]
        pos += dim


def test_unit_test_mapping_on_the_oracle(oracle, noise):
    """CPU: the mapped circuits, run by the oracle as pure states, give the unit tests'
    expected rho = |psi><psi| (vector index i + 2^n j) within ERROR_BAR: the mapping
    itself is right before the GPU is involved."""
    failed = []
    for name, n, gl, er, ei in kat_circuits(noise):
        arr = G.to_array(gl) if gl else np.zeros(0, dtype=G.GATE_DTYPE)
        re, im = oracle.run(n, arr)
        psi = re + 1j * im
        vec = np.outer(psi, psi.conj()).T.reshape(-1)
        if np.max(np.abs(vec.real - er)) > 1e-3 or np.max(np.abs(vec.imag - ei)) > 1e-3:
            failed.append(name)
    assert not failed, failed
