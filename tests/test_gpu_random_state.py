"""Every engine on a random input state (svb_set_state_soa), against the oracle applied to the
same state.  From |0..0> an op that only multiplies amplitudes with some qubit at 1 (a phase on
a qubit that is not local in the pass, a tile-selected block variant, a per-tile condition)
acts on zeros, so a kernel or plan that mishandles it passes every test that starts there;
these circuits are heavy in such ops, and the ansatz segments open with runs of RZ on qubits
that are not local in the first pass."""
import numpy as np
import pytest

from svsim_b200 import circuits, gates as G

pytestmark = pytest.mark.gpu


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    s = rng.normal(size=(2, 1 << n))
    s /= np.sqrt((s ** 2).sum())
    return s[0].copy(), s[1].copy()


def diagonal_heavy(n, m, seed, srn=False):
    rng = np.random.default_rng(seed)
    gl = []
    for _ in range(m):
        r = rng.random()
        q = int(rng.integers(n))
        q2 = int(rng.integers(n - 1))
        q2 += q2 >= q
        if r < 0.25:
            gl.append(G.RZ(rng.uniform(-3, 3), q))
        elif r < 0.35:
            gl.append(G.T(q))
        elif r < 0.45:
            gl.append(G.U1(rng.uniform(-3, 3), q))
        elif r < 0.6:
            gl.append(G.CX(q, q2))
        elif r < 0.7:
            gl.append(G.CZ(q, q2))
        elif r < 0.75:
            gl.append(G.CRZ(rng.uniform(-3, 3), q, q2))
        elif r < 0.85:
            gl.append(G.RY(rng.uniform(-3, 3), q))
        else:
            gl.append(G.U3(*rng.uniform(-3, 3, 3), q))
    if srn:
        gl.append(G.SRN(0))
    return G.to_array(gl)


def ansatz_segment(n, lo, hi):
    pc = circuits.hardware_efficient_ansatz(n=n, layers=2, seed=7)
    return np.ascontiguousarray(pc.evaluated(pc.params)[lo:hi])


CASES = [(14, diagonal_heavy(14, 120, 1)), (17, diagonal_heavy(17, 150, 2)),
         (20, ansatz_segment(20, 24, 48)), (20, ansatz_segment(20, 72, 96))]


def run_on(nat, n, g, state, precision, engine, tile=0, k=0):
    h = nat.Handle(n, 0, precision)
    h.set_engine(engine, tile, k)
    h.set_state(*state)
    h.set_circuit(g)
    h.run()
    h.sync()
    re, im = h.get_state()
    h.close()
    return re + 1j * im


@pytest.mark.parametrize("case", range(len(CASES)))
def test_fp64_engines_on_random_state(oracle, case):
    from svsim_b200 import _native as nat
    n, g = CASES[case]
    st = random_state(n, 100 + case)
    ore, oim = oracle.run(n, g, state=st)
    want = ore + 1j * oim
    for engine, tile in ((nat.ENGINE_PAIRS, 0), (nat.ENGINE_STAGED, 10), (nat.ENGINE_STAGED, 12),
                         (nat.ENGINE_PER_GATE, 0)):
        got = run_on(nat, n, g, st, nat.SVB_FP64, engine, tile)
        assert np.max(np.abs(got - want)) <= 1e-12, (engine, tile)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_fused_engine_on_random_state(oracle, case):
    from svsim_b200 import _native as nat
    n, g = CASES[case]
    st = random_state(n, 200 + case)
    ore, oim = oracle.run(n, g, state=st)
    want = ore + 1j * oim
    for k in (3, 4, 5, 6):
        got = run_on(nat, n, g, st, nat.SVB_FP32, nat.ENGINE_FUSED, 0, k)
        f = abs(np.vdot(want, got)) ** 2 / (np.vdot(got, got).real * np.vdot(want, want).real)
        assert 1 - f <= 1e-6, k


def test_srn_circuit_on_random_state(oracle):
    """SRN (not a matrix) keeps a circuit on the staged and per-gate engines."""
    from svsim_b200 import _native as nat
    n = 15
    g = diagonal_heavy(n, 100, 9, srn=True)
    st = random_state(n, 9)
    ore, oim = oracle.run(n, g, state=st)
    want = ore + 1j * oim
    for engine, tile in ((nat.ENGINE_STAGED, 11), (nat.ENGINE_PER_GATE, 0)):
        got = run_on(nat, n, g, st, nat.SVB_FP64, engine, tile)
        assert np.max(np.abs(got - want)) <= 1e-12, engine


def test_batched_pairs_on_segments(oracle):
    """The batch's pair-engine path on the same segments (from |0..0>, with a prefix that
    spreads the state first) against the oracle."""
    from svsim_b200 import _native as nat
    n = 20
    prep = G.to_array([G.U3(0.3 + 0.1 * q, 0.2, -0.4, q) for q in range(n)])
    batch = [(n, np.concatenate([prep, ansatz_segment(n, lo, hi)])) for lo, hi in ((24, 48), (72, 96))]
    b = nat.CircuitBatch(batch, tile_bits=nat.CBATCH_PAIRS)
    assert b.info().pair_circuits == 2
    b.run()
    for i, (nn, g) in enumerate(batch):
        re, im = oracle.run(nn, g)
        assert np.max(np.abs(b.state(i) - (re + 1j * im))) <= 1e-12, i
    b.close()


def every_op_circuit(n, reps, seed, srn):
    """All 38 ops of the reference, shuffled, on random qubits (SRN and the non-unitary R
    only where asked: the pair engine takes matrices only)."""
    import math
    rng = np.random.default_rng(seed)
    gl = []
    for _ in range(reps):
        names = list(G.OP_NAMES)
        rng.shuffle(names)
        for name in names:
            if name == "SRN" and not srn:
                continue
            qs = [int(x) for x in rng.permutation(n)[:G.N_QUBITS[name]]]
            npar = {"U3": 3, "U2": 2, "CU3": 3}.get(name, 1 if name in (
                "U1", "RX", "RY", "RZ", "CRX", "CRY", "CRZ", "CU1", "RXX", "RZZ", "RYY", "R") else 0)
            gl.append(G.FACTORIES[name](*([rng.uniform(-math.pi, math.pi) for _ in range(npar)] + qs)))
    return G.to_array(gl)


@pytest.mark.parametrize("n,seed", [(12, 1), (15, 2), (17, 3), (21, 4)])
def test_every_op_every_engine_on_random_state(oracle, n, seed):
    """Differential check: every op, every FP64 engine, a random input state, the oracle."""
    from svsim_b200 import _native as nat
    g = every_op_circuit(n, 3, seed, srn=False)
    st = random_state(n, 300 + seed)
    ore, oim = oracle.run(n, g, state=st)
    want = ore + 1j * oim
    for engine, tile in ((nat.ENGINE_PAIRS, 0), (nat.ENGINE_STAGED, 10), (nat.ENGINE_STAGED, 11),
                         (nat.ENGINE_STAGED, 12), (nat.ENGINE_PER_GATE, 0)):
        got = run_on(nat, n, g, st, nat.SVB_FP64, engine, tile)
        assert np.max(np.abs(got - want)) <= 1e-12, (engine, tile)
    for k in (4, 5, 6):
        got = run_on(nat, n, g, st, nat.SVB_FP32, nat.ENGINE_FUSED, 0, k)
        f = abs(np.vdot(want, got)) ** 2 / (np.vdot(got, got).real * np.vdot(want, want).real)
        assert 1 - f <= 1e-6, k
