"""Batched circuits (svb_cbatch_*): circuits of uneven qubit counts run together by one
persistent, graph-replayed launch (two with the pair engine), each checked against the
oracle (state and Pauli-sum energy), with the tile and block sizes and the engine chosen by
the autotuner or given."""
import numpy as np
import pytest

from svsim_b200 import circuits, gates as G

pytestmark = pytest.mark.gpu


def native():
    from svsim_b200 import _native
    return _native


def mixed_batch(seed=0, count=20, lo=10, hi=22):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(lo, hi + 1))
        depth = 6 if n <= 16 else 3
        g = circuits.random_matching_circuit(n, depth, seed=seed * 100 + i)
        if i % 3 == 0:                      # composites, diagonal ops and SRN as well
            extra = [G.CCX(0, 1, 2), G.CRZ(0.4, 1, n - 1), G.T(n - 1), G.RZZ(0.3, 0, n - 2),
                     G.SRN(3), G.CSWAP(n - 1, 2, 5), G.S(n - 2), G.CU3(0.1, 0.2, 0.3, n - 3, 4)]
            g = np.concatenate([g, G.to_array(extra)])
        out.append((n, g))
    return out


@pytest.mark.parametrize("precision,tile_bits", [(0, 0), (0, 10), (1, 0), (0, -1)])
def test_mixed_batch_matches_oracle(oracle, precision, tile_bits):
    """tile_bits -1 (CBATCH_PAIRS): the FP64 circuits of 12 or more qubits without SRN on
    the pair engine, the others (n = 10, 11, and those with SRN) on the sweep."""
    nat = native()
    batch = mixed_batch(seed=1 + precision + abs(tile_bits))
    terms = [circuits.zz_x_hamiltonian(n) for n, _ in batch]
    terms[2] = None                          # a circuit without an observable
    b = nat.CircuitBatch(batch, terms, precision=precision, tile_bits=tile_bits)
    info = b.info()
    assert info.tuned == (1 if tile_bits == 0 else 0)
    if tile_bits == nat.CBATCH_PAIRS:
        eligible = sum(1 for i, (n, g) in enumerate(batch) if n >= 12 and i % 3 != 0)
        assert info.pair_circuits == eligible and 0 < eligible < len(batch)
        assert info.pair_phases > 0 and info.pair_grid > 0
    e = b.run()
    e2 = b.run()
    assert np.array_equal(e, e2)             # fixed-order sums: repeatable
    for i, (n, g) in enumerate(batch):
        re, im = oracle.run(n, g)
        a = b.state(i)
        ref = re + 1j * im
        if precision == 0:
            assert np.max(np.abs(a - ref)) <= 1e-12, i
        else:
            f = abs(np.vdot(ref, a)) ** 2 / (np.vdot(a, a).real * np.vdot(ref, ref).real)
            assert 1 - f <= 1e-6, i
        want = oracle.expectation(n, re, im, terms[i]) if terms[i] is not None else 0.0
        assert abs(e[i] - want) <= (1e-12 if precision == 0 else 1e-4) * max(1.0, abs(want)), i
    b.close()


def test_small_circuits_and_single_tiles(oracle):
    nat = native()
    batch = []
    for n in range(1, 13):
        g = circuits.random_matching_circuit(n, 4, seed=n)
        batch.append((n, g))
    b = nat.CircuitBatch(batch, tile_bits=12)
    b.run()
    for i, (n, g) in enumerate(batch):
        re, im = oracle.run(n, g)
        assert np.max(np.abs(b.state(i) - (re + 1j * im))) <= 1e-12, n
    b.close()


@pytest.mark.parametrize("tile_bits", [0, -1])
def test_parameter_sets_with_new_angles(oracle, tile_bits):
    """64 parameter points of one ansatz in one launch; new angles for the same structure
    through svb_cbatch_run(gates) (on the pair engine: new gate fragments for the same
    blocks), against the oracle's energies."""
    nat = native()
    pc = circuits.hardware_efficient_ansatz(n=12, layers=4, seed=2)
    terms = circuits.zz_x_hamiltonian(pc.n)
    pts = np.random.default_rng(4).uniform(-np.pi, np.pi, size=(64, len(pc.params)))
    batch = [(pc.n, pc.evaluated(p)) for p in pts]
    b = nat.CircuitBatch(batch, [terms] * len(batch), tile_bits=tile_bits)
    if tile_bits == nat.CBATCH_PAIRS:
        assert b.info().pair_circuits == 64
    e = b.run()
    for i in (0, 17, 63):
        re, im = oracle.run(pc.n, batch[i][1])
        assert abs(e[i] - oracle.expectation(pc.n, re, im, terms)) <= 1e-12
    pts2 = pts[::-1].copy()
    e2 = b.run(np.concatenate([pc.evaluated(p) for p in pts2]))
    assert np.allclose(e2, e[::-1], atol=1e-12, rtol=0)
    b.close()


def test_invalid_batches_rejected():
    nat = native()
    with pytest.raises(nat.SvbError):
        nat.CircuitBatch([(25, circuits.random_matching_circuit(25, 1, seed=0))])
    with pytest.raises(nat.SvbError):
        nat.CircuitBatch([(4, G.to_array([G.CX(0, 4)]))])
    b = nat.CircuitBatch([(5, circuits.random_matching_circuit(5, 2, seed=1))], tile_bits=8)
    g = circuits.random_matching_circuit(5, 2, seed=1)
    g["qb"][0][0] = (g["qb"][0][0] + 1) % 5        # another structure
    with pytest.raises(nat.SvbError):
        b.run(g)
    b.close()


@pytest.mark.parametrize("n,precision", [(14, 0), (22, 0), (20, 1)])
def test_autotune_single_circuit(oracle, n, precision):
    """svb_autotune times the candidate engines, AUTO then uses the choice for circuits of
    the same structure (other angles included), and results stay correct."""
    nat = native()
    g = circuits.random_matching_circuit(n, 6, seed=n)
    h = nat.Handle(n, 0, precision)
    r = h.autotune(g)
    assert r.candidates >= 2 and r.best_ms > 0
    assert r.best_ms <= r.default_ms * 1.5 or r.default_ms < 0      # timing noise at small n
    info = h.plan_info()
    assert info.engine == r.engine
    g2 = circuits.random_matching_circuit(n, 6, seed=n)
    g2["theta"] += 0.1                          # same structure, other angles
    h.set_circuit(g2)
    assert h.plan_info().engine == r.engine
    h.run()
    h.sync()
    re, im = h.get_state()
    ore, oim = oracle.run(n, g2)
    a, b = re + 1j * im, ore + 1j * oim
    if precision == 0:
        assert np.max(np.abs(a - b)) <= 1e-12
    else:
        assert 1 - abs(np.vdot(b, a)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real) <= 1e-6
    h.close()


def test_pair_engine_request_on_fp32_and_small_circuits(oracle):
    """CBATCH_PAIRS where the pair engine cannot run (FP32, n < 12, SRN) keeps every circuit
    on the shared-memory sweep, with the same results."""
    nat = native()
    batch = [(n, circuits.random_matching_circuit(n, 4, seed=40 + n)) for n in (8, 11, 13)]
    b = nat.CircuitBatch(batch, precision=1, tile_bits=nat.CBATCH_PAIRS)
    assert b.info().pair_circuits == 0
    b.run()
    for i, (n, g) in enumerate(batch):
        re, im = oracle.run(n, g)
        a = b.state(i)
        ref = re + 1j * im
        f = abs(np.vdot(ref, a)) ** 2 / (np.vdot(a, a).real * np.vdot(ref, ref).real)
        assert 1 - f <= 1e-6, n
    b.close()
    srn = [(13, np.concatenate([circuits.random_matching_circuit(13, 3, seed=7), G.to_array([G.SRN(2)])]))]
    b = nat.CircuitBatch(srn, tile_bits=nat.CBATCH_PAIRS)
    assert b.info().pair_circuits == 0
    b.run()
    re, im = oracle.run(13, srn[0][1])
    assert np.max(np.abs(b.state(0) - (re + 1j * im))) <= 1e-12
    b.close()
