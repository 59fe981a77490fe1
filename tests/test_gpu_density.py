"""Density matrices with noise (svb_dm_*): rho -> U rho U^dagger per gate and a Kraus
channel on each touched qubit, against a numpy density-matrix restatement built from
the oracle's gate unitaries, on both engines the superoperator blocks run on."""
import numpy as np
import pytest

from svsim_b200 import circuits, density as D, gates as G

pytestmark = pytest.mark.gpu


def gate_unitary(oracle, n, g):
    """Full 2^n x 2^n unitary of one gate record, column k = the oracle applied to |k>."""
    d = 1 << n
    u = np.zeros((d, d), dtype=complex)
    arr = np.array([g], dtype=G.GATE_DTYPE)
    for k in range(d):
        re = np.zeros(d)
        im = np.zeros(d)
        re[k] = 1.0
        r2, i2 = oracle.run(n, arr, state=(re, im))
        u[:, k] = r2 + 1j * i2
    return u


def on_qubit(n, q, k):
    """k (2x2) on qubit q of n (little-endian: qubit 0 is the lowest index bit)."""
    out = np.eye(1)
    for j in reversed(range(n)):
        out = np.kron(out, k if j == q else np.eye(2))
    return out


def rho_reference(oracle, n, gates, kraus=None):
    d = 1 << n
    rho = np.zeros((d, d), dtype=complex)
    rho[0, 0] = 1.0
    for g in gates:
        u = gate_unitary(oracle, n, g)
        rho = u @ rho @ u.conj().T
        if kraus:
            name = G.OP_NAMES[int(g["op"])]
            for q in [int(x) for x in g["qb"][:G.N_QUBITS[name]]]:
                ks = [on_qubit(n, q, np.asarray(k, dtype=complex)) for k in kraus]
                rho = sum(k @ rho @ k.conj().T for k in ks)
    return rho


@pytest.mark.parametrize("n,channel", [(5, None), (5, "dp"), (6, "ad"), (7, "dp")])
def test_density_matrix_matches_numpy(oracle, n, channel):
    kraus = {None: None, "dp": D.depolarizing(0.02), "ad": D.amplitude_damping(0.05)}[channel]
    gates = circuits.random_matching_circuit(n, 3, seed=n)
    gates = np.concatenate([gates, G.to_array([G.CCX(0, 1, 2), G.CRY(0.3, 1, 3), G.RZZ(0.7, 0, 4)])])
    dm = D.DensityMatrix(n)
    dm.set_circuit(gates, kraus)
    dm.run()
    rho = dm.rho()
    ref = rho_reference(oracle, n, gates, kraus)
    assert np.max(np.abs(rho - ref)) <= 1e-12
    p = dm.probabilities()
    assert np.max(np.abs(p - np.real(np.diag(ref)))) <= 1e-12
    assert abs(p.sum() - 1.0) <= 1e-12
    # the pair engine runs the blocks from 2n = 12 qubits on
    assert dm.plan_info().engine == (4 if 2 * n >= 12 else 1)
    dm.close()


def test_pure_state_is_the_state_vector_outer_product(oracle):
    n = 9
    gates = circuits.random_matching_circuit(n, 6, seed=4)
    dm = D.DensityMatrix(n)
    dm.set_circuit(gates)
    dm.run()
    re, im = oracle.run(n, gates)
    psi = re + 1j * im
    assert np.max(np.abs(dm.rho() - np.outer(psi, psi.conj()))) <= 1e-12
    u = np.random.default_rng(2).random(4096)
    samples = dm.measure(u)
    ref, _ = oracle.measure(n, re, im, u)
    assert np.array_equal(samples, ref)
    dm.close()


def test_noise_reduces_purity_and_srn_is_rejected():
    from svsim_b200 import _native as nat
    n = 6
    gates = circuits.random_matching_circuit(n, 4, seed=1)
    dm = D.DensityMatrix(n)
    dm.set_circuit(gates, D.depolarizing(0.05))
    dm.run()
    purity = dm.handle.norm2()                      # Tr(rho^2)
    assert purity < 0.9 and abs(dm.probabilities().sum() - 1) <= 1e-12
    with pytest.raises(nat.SvbError):
        dm.set_circuit(G.to_array([G.SRN(0)]))
    dm.close()
