"""Parity of the CUDA path (through the C ABI) with the reference: golden fixtures made by
the reference's CPU backend, and the C oracle on seeded circuits.

Bars: FP64 1-F <= 1e-12 and max |d amp| <= 1e-12 (in practice ~1e-15); samples
bit-identical to the reference's own measure() given the same uniform draws; FP32
1-F <= 1e-6."""
import math

import numpy as np
import pytest

from conftest import cx_dense_circuit, fidelity, load_golden
from svsim_b200 import circuits, gates as G

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def native():
    from svsim_b200 import _native
    return _native


def run_gpu(n, gates, engine=0, tile_bits=0, precision=0, state=None):
    nat = native()
    h = nat.Handle(n, 0, precision)
    h.set_engine(engine, tile_bits, 0)
    if state is not None:
        h.set_state(*state)
    h.set_circuit(gates)
    h.run()
    h.sync()
    re, im = h.get_state()
    return h, re, im


def engines_for(n, precision=0):
    nat = native()
    out = [(nat.ENGINE_PER_GATE, 0)]
    tiles = (10, 11, 12) if precision == 0 else (11, 12, 13)
    out += [(nat.ENGINE_STAGED, m) for m in tiles if m <= n]
    return out


def assert_close(re, im, ore, oim, tol=FP64_TOL):
    a = re + 1j * im
    b = ore + 1j * oim
    assert np.max(np.abs(a - b)) <= tol, np.max(np.abs(a - b))
    if np.vdot(b, b).real > 0:
        assert 1 - fidelity(a, b) <= tol


def mixed_circuit(n, reps, seed):
    rng = np.random.default_rng(seed)
    gl = G.from_array(circuits.random_matching_circuit(n, 1, seed=seed))
    for _ in range(reps):
        for name in G.OP_NAMES:
            qs = [int(x) for x in rng.permutation(n)[:G.N_QUBITS[name]]]
            npar = {"U3": 3, "U2": 2, "CU3": 3}.get(name, 1 if name in (
                "U1", "RX", "RY", "RZ", "CRX", "CRY", "CRZ", "CU1", "RXX", "RZZ", "RYY", "R") else 0)
            gl.append(G.FACTORIES[name](*([rng.uniform(-math.pi, math.pi) for _ in range(npar)] + qs)))
    return G.to_array(gl)


def inverse_circuit(gates):
    """U^dagger of a U3/CX circuit: U3(t,p,l)^-1 = U3(-t,-l,-p), CX^-1 = CX."""
    inv = gates[::-1].copy()
    u3 = inv["op"] == G.OP["U3"]
    th, ph, la = inv["theta"][u3].copy(), inv["phi"][u3].copy(), inv["lam"][u3].copy()
    inv["theta"][u3], inv["phi"][u3], inv["lam"][u3] = -th, -la, -ph
    return inv


# ---- known answers and golden fixtures --------------------------------------------------

def test_kat_known_answers():
    k = load_golden("kat.npz")
    pos = 0
    for i, name in enumerate(k["names"]):
        n = int(k["n"][i])
        g = k["gates"][k["gate_offsets"][i]:k["gate_offsets"][i + 1]]
        _, re, im = run_gpu(n, g)
        dim = 1 << n
        assert np.all(np.abs(re - k["expected_re"][pos:pos + dim]) <= 1e-3), name
        assert np.all(np.abs(im - k["expected_im"][pos:pos + dim]) <= 1e-3), name
        assert_close(re, im, k["ref_re"][pos:pos + dim], k["ref_im"][pos:pos + dim], 1e-15)
        pos += dim


def test_every_op_matches_reference_states():
    d = load_golden("all_ops_n6.npz")
    for i, name in enumerate(d["names"]):
        g = d["gates"][d["gate_offsets"][i]:d["gate_offsets"][i + 1]]
        _, re, im = run_gpu(6, g)
        assert np.max(np.abs(re - d["re"][i])) <= 1e-14, name
        assert np.max(np.abs(im - d["im"][i])) <= 1e-14, name


def test_per_gate_engine_is_bit_identical_to_the_reference_cpu():
    """The per-gate engine is compiled without FMA contraction and evaluates the reference's
    gate expressions in the reference's order, so its FP64 states equal the reference CPU
    backend's bit for bit: every op (golden states of svsim_cpu_sin.hpp) and the 14 unit
    tests' circuits."""
    nat = native()
    d = load_golden("all_ops_n6.npz")
    bad = []
    for i, name in enumerate(d["names"]):
        g = d["gates"][d["gate_offsets"][i]:d["gate_offsets"][i + 1]]
        _, re, im = run_gpu(6, g, nat.ENGINE_PER_GATE)
        if not (np.array_equal(re, d["re"][i]) and np.array_equal(im, d["im"][i])):
            bad.append(str(name))
    assert not bad, sorted(set(bad))
    b = load_golden("brickwork.npz")
    _, re, im = run_gpu(12, b["gates12"], nat.ENGINE_PER_GATE)
    assert np.array_equal(re, b["re12"]) and np.array_equal(im, b["im12"])


@pytest.mark.parametrize("n", [13, 21])
def test_per_gate_engine_is_bit_identical_to_the_oracle(oracle, n):
    nat = native()
    g = mixed_circuit(n, 2, seed=n)
    ore, oim = oracle.run(n, g)
    _, re, im = run_gpu(n, g, nat.ENGINE_PER_GATE)
    assert np.array_equal(re, ore) and np.array_equal(im, oim)


@pytest.mark.parametrize("engine_idx", range(4))
def test_every_op_all_engines(oracle, engine_idx):
    n = 12
    engines = engines_for(n)
    engine, tile = engines[engine_idx]
    g = mixed_circuit(n, 4, seed=engine_idx)
    _, re, im = run_gpu(n, g, engine, tile)
    ore, oim = oracle.run(n, g)
    assert_close(re, im, ore, oim)


@pytest.mark.parametrize("engine_idx", range(4))
def test_brickwork_470_gates_and_samples(engine_idx):
    """The 470-gate brickwork circuit at n=16: amplitudes and checksum against the
    reference's state, 1-F, and the 1024 samples of the reference's own measure()."""
    d = load_golden("brickwork.npz")
    engine, tile = engines_for(16)[engine_idx]
    h, re, im = run_gpu(16, d["gates16"], engine, tile)
    idx = d["idx16"]
    assert np.max(np.abs(re[idx] - d["re16_at"])) <= FP64_TOL
    assert np.max(np.abs(im[idx] - d["im16_at"])) <= FP64_TOL
    i = np.arange(1 << 16, dtype=np.float64)
    w = np.cos(0.7 * i) + 1j * np.sin(1.3 * i)
    assert abs(np.sum((re + 1j * im) * w) - d["checksum16"][0]) <= 1e-10
    samples, total = h.measure(d["uniforms16"])
    assert np.array_equal(samples, d["samples16"])
    assert abs(total - d["norm16"][0]) <= 1e-12
    _, re12, im12 = run_gpu(12, d["gates12"], engine if tile <= 12 else 1, tile)
    assert_close(re12, im12, d["re12"], d["im12"])


def test_matching_golden():
    d = load_golden("matching_n12.npz")
    for engine, tile in engines_for(12):
        _, re, im = run_gpu(12, d["gates"], engine, tile)
        assert_close(re, im, d["re"], d["im"])


@pytest.mark.parametrize("n", [14, 20])
def test_random_matching_vs_oracle(oracle, n):
    g = circuits.random_matching_circuit(n, 8, seed=n)
    ore, oim = oracle.run(n, g)
    for engine, tile in engines_for(n):
        _, re, im = run_gpu(n, g, engine, tile)
        assert_close(re, im, ore, oim)


def test_from_arbitrary_state(oracle):
    n = 13
    rng = np.random.default_rng(3)
    st = (rng.standard_normal(1 << n), rng.standard_normal(1 << n))
    g = mixed_circuit(n, 2, seed=4)
    ore, oim = oracle.run(n, g, state=st)
    for engine, tile in engines_for(n):
        _, re, im = run_gpu(n, g, engine, tile, state=st)
        assert np.max(np.abs(re - ore)) <= 1e-11 and np.max(np.abs(im - oim)) <= 1e-11


def test_fp32_engines(oracle):
    n = 14
    g = mixed_circuit(n, 2, seed=8)
    ore, oim = oracle.run(n, g)
    for engine, tile in engines_for(n, precision=1):
        _, re, im = run_gpu(n, g, engine, tile, precision=1)
        assert 1 - fidelity(re + 1j * im, ore + 1j * oim) <= 1e-6


# ---- measurement ------------------------------------------------------------------------

def test_measure_rules(oracle):
    nat = native()
    h = nat.Handle(3, 0, nat.SVB_FP64)
    h.set_circuit(G.to_array([G.X(0), G.X(2)]))
    h.run()
    s, tot = h.measure(np.array([0.0, 0.5, 0.999999, 1.0, -0.1]))
    assert list(s) == [5, 5, 5, 0, 0] and tot == 1.0
    # uniform superposition: boundaries
    h2 = nat.Handle(2, 0, nat.SVB_FP64)
    h2.set_circuit(G.to_array([G.H(0), G.H(1)]))
    h2.run()
    u = np.array([0.0, 0.2499, 0.25000001, 0.5000001, 0.75000001, 0.9999])
    s, _ = h2.measure(u)
    re, im = h2.get_state()
    want, _ = oracle.measure(2, re, im, u)
    assert list(s) == list(want) == [0, 0, 1, 2, 3, 3]


@pytest.mark.parametrize("n", [5, 12, 17, 21])
def test_measure_matches_oracle_rule(oracle, n):
    g = circuits.random_matching_circuit(n, 4, seed=n)
    h, re, im = run_gpu(n, g)
    u = np.random.default_rng(n).random(4096)
    s, tot = h.measure(u)
    want, wtot = oracle.measure(n, re, im, u)
    assert np.array_equal(s, want)
    assert abs(tot - wtot) <= 1e-12


def test_measure_seeded_reproduces_reference_samples():
    """svb_measure_seeded(seed) draws the reference's rand()/RAND_MAX sequence after
    srand(seed): on the 470-gate brickwork state it returns the samples the reference's
    own measure() gave for that seed (golden fixture), on every engine."""
    d = load_golden("brickwork.npz")
    seed = int(d["sample_seed"][0])
    for engine, tile in engines_for(16):
        h, _, _ = run_gpu(16, d["gates16"], engine, tile)
        samples, total = h.measure_seeded(seed, 1024)
        assert np.array_equal(samples, d["samples16"])
        assert abs(total - d["norm16"][0]) <= 1e-12
        again, _ = h.measure_seeded(seed, 1024)
        assert np.array_equal(again, samples)
    empty, _ = h.measure_seeded(seed, 0)
    assert len(empty) == 0


def test_norm_of_non_unitary_circuit(oracle):
    """SRN and R are not norm-preserving as coded in the reference."""
    n = 10
    g = G.to_array([G.H(3), G.SRN(2), G.R(0.7, 4), G.SRN(9)])
    h, re, im = run_gpu(n, g)
    ore, oim = oracle.run(n, g)
    assert_close(re, im, ore, oim)
    assert abs(h.norm2() - np.sum(ore ** 2 + oim ** 2)) <= 1e-14


def test_expectation(oracle):
    n = 12
    g = circuits.random_matching_circuit(n, 3, seed=2)
    h, re, im = run_gpu(n, g)
    terms = circuits.zz_x_hamiltonian(n)
    assert abs(h.expectation(terms) - oracle.expectation(n, re, im, terms)) <= 1e-12


# ---- API behaviour ------------------------------------------------------------------------

def test_state_persists_across_runs_and_reset(oracle):
    nat = native()
    n = 11
    g1 = circuits.random_matching_circuit(n, 2, seed=1)
    g2 = circuits.random_matching_circuit(n, 2, seed=2)
    h = nat.Handle(n, 0, nat.SVB_FP64)
    h.set_circuit(g1)
    h.run()
    h.clear_circuit()            # the state stays, as Simulation::clear_circuit (:341-358)
    h.set_circuit(g2)
    h.run()
    re, im = h.get_state()
    ore, oim = oracle.run(n, np.concatenate([g1, g2]))
    assert_close(re, im, ore, oim)
    h.run()                      # the same circuit again continues from the state
    ore, oim = oracle.run(n, g2, state=(ore, oim))
    re, im = h.get_state()
    assert_close(re, im, ore, oim)
    h.reset()
    re, im = h.get_state()
    assert re[0] == 1.0 and np.count_nonzero(re) == 1 and not im.any()


def test_invalid_inputs_rejected():
    nat = native()
    h = nat.Handle(4, 0, nat.SVB_FP64)
    bad = [G.to_array([G.CX(1, 1)]), G.to_array([G.H(4)]), G.to_array([G.CCX(0, 2, 0)])]
    arr = G.to_array([G.H(0)])
    arr["op"][0] = 38
    bad.append(arr)
    for g in bad:
        with pytest.raises(nat.SvbError) as e:
            h.set_circuit(g)
        assert e.value.status == nat.SVB_ERR_INVALID
    h.clear_circuit()
    with pytest.raises(nat.SvbError) as e:
        h.run()
    assert e.value.status == nat.SVB_ERR_STATE
    with pytest.raises(nat.SvbError):
        nat.Handle(36, 0, nat.SVB_FP64)       # 1 TiB: out of memory, reported not fatal


def test_empty_and_identity_circuits():
    nat = native()
    h = nat.Handle(12, 0, nat.SVB_FP64)
    h.set_circuit(np.zeros(0, dtype=G.GATE_DTYPE))
    h.run()
    h.set_circuit(G.to_array([G.ID(3), G.ID(0)]))
    h.run()
    re, im = h.get_state()
    assert re[0] == 1.0 and np.count_nonzero(re) == 1


def test_python_simulation_api(oracle):
    from svsim_b200 import Simulation
    sim = Simulation(10, 0)
    sim.append(Simulation.X(1))
    sim.append(Simulation.X(5))
    sim.upload()
    sim.run()
    sim.clear_circuit()
    for a, b, c in [(0, 5, 1), (1, 6, 2)]:
        sim.append(Simulation.CX(c, b))
        sim.append(Simulation.CX(c, a))
        sim.append(Simulation.CCX(a, b, c))
    sim.upload()
    sim.run()
    res = sim.measure(10)
    assert len(res) == 10 and all(0 <= r < 1024 for r in res)
    with pytest.raises(ValueError):
        sim.append(Simulation.H(10))


# ---- large states: size-independent properties ---------------------------------------------

@pytest.mark.parametrize("n", [26, 31])
def test_mirror_circuit_returns_to_zero(n):
    """C then C^dagger must give back |0..0>; at n=31 indices pass 2^31 (32 GiB FP64)."""
    nat = native()
    g = circuits.random_matching_circuit(n, 3, seed=n)
    mirror = np.concatenate([g, inverse_circuit(g)])
    h = nat.Handle(n, 0, nat.SVB_FP64)
    h.set_circuit(mirror)
    h.run()
    h.sync()
    u = np.array([0.3, 0.999999999])
    s, tot = h.measure(u)
    assert abs(tot - 1.0) <= 1e-12
    assert list(s) == [0, 0]          # all probability on |0..0>
    h.set_circuit(g)
    h.run()
    assert abs(h.norm2() - 1.0) <= 1e-12


def test_staged_equals_per_gate_at_n26():
    nat = native()
    n = 26
    g = circuits.random_matching_circuit(n, 4, seed=11)
    _, re1, im1 = run_gpu(n, g, nat.ENGINE_PER_GATE)
    _, re2, im2 = run_gpu(n, g, nat.ENGINE_STAGED, 12)
    assert np.max(np.abs(re1 - re2)) <= 1e-13 and np.max(np.abs(im1 - im2)) <= 1e-13


# ---- pair engine (FP64 two-qubit blocks on the FP64 tensor cores) ---------------------

def no_srn(g):
    return g[g["op"] != G.OP["SRN"]]


def test_pair_engine_brickwork_golden_and_samples():
    """The 470-gate brickwork circuit at n=16 through the pair engine: amplitudes and
    checksum against the reference's state and the 1024 samples of its own measure()."""
    nat = native()
    d = load_golden("brickwork.npz")
    h, re, im = run_gpu(16, d["gates16"], nat.ENGINE_PAIRS)
    assert h.plan_info().engine == nat.ENGINE_PAIRS
    idx = d["idx16"]
    assert np.max(np.abs(re[idx] - d["re16_at"])) <= FP64_TOL
    assert np.max(np.abs(im[idx] - d["im16_at"])) <= FP64_TOL
    i = np.arange(1 << 16, dtype=np.float64)
    w = np.cos(0.7 * i) + 1j * np.sin(1.3 * i)
    assert abs(np.sum((re + 1j * im) * w) - d["checksum16"][0]) <= 1e-10
    samples, total = h.measure(d["uniforms16"])
    assert np.array_equal(samples, d["samples16"])
    assert abs(total - d["norm16"][0]) <= 1e-12


@pytest.mark.parametrize("n", [12, 14, 17, 20, 22])
def test_pair_engine_random_matching_vs_oracle(oracle, n):
    nat = native()
    g = circuits.random_matching_circuit(n, 8, seed=n + 1)
    ore, oim = oracle.run(n, g)
    _, re, im = run_gpu(n, g, nat.ENGINE_PAIRS)
    assert_close(re, im, ore, oim)


def test_pair_engine_pass_with_gates_beyond_shared_memory(oracle):
    """The CX-dense n = 12 circuit: its passes hold more gate fragments than fit beside the
    tile in shared memory (tests/test_plan.py checks that the plan says so), so the kernel
    reads those passes' gates from global memory."""
    nat = native()
    g = cx_dense_circuit()
    ore, oim = oracle.run(12, g)
    _, re, im = run_gpu(12, g, nat.ENGINE_PAIRS)
    assert_close(re, im, ore, oim)


@pytest.mark.parametrize("n", [12, 15])
def test_pair_engine_every_op_but_srn(oracle, n):
    nat = native()
    g = no_srn(mixed_circuit(n, 4, seed=n))
    ore, oim = oracle.run(n, g)
    _, re, im = run_gpu(n, g, nat.ENGINE_PAIRS)
    assert_close(re, im, ore, oim)


def test_pair_engine_from_arbitrary_state_and_qaoa(oracle):
    nat = native()
    n = 13
    rng = np.random.default_rng(3)
    st = (rng.standard_normal(1 << n), rng.standard_normal(1 << n))
    g = no_srn(mixed_circuit(n, 2, seed=4))
    ore, oim = oracle.run(n, g, state=st)
    _, re, im = run_gpu(n, g, nat.ENGINE_PAIRS, state=st)
    assert np.max(np.abs(re - ore)) <= 1e-11 and np.max(np.abs(im - oim)) <= 1e-11
    q = circuits.qaoa_instances(1, n_min=16, n_max=16, seed=9)[0].circuit()
    ore, oim = oracle.run(16, q)
    _, re, im = run_gpu(16, q, nat.ENGINE_PAIRS)
    assert_close(re, im, ore, oim)


def test_pair_engine_matches_staged_on_device():
    nat = native()
    n = 26
    g = circuits.random_matching_circuit(n, 12, seed=77)
    ha = nat.Handle(n, 0, nat.SVB_FP64)
    ha.set_engine(nat.ENGINE_PAIRS, 0, 0)
    ha.set_circuit(g)
    ha.run()
    hb = nat.Handle(n, 0, nat.SVB_FP64)
    hb.set_engine(nat.ENGINE_STAGED, 12, 0)
    hb.set_circuit(g)
    hb.run()
    f, d = ha.compare(hb)
    assert 1 - f <= 1e-12 and d <= 1e-13


def test_pair_engine_rejects_srn_fp32_and_small_states():
    nat = native()
    h = nat.Handle(12, 0, nat.SVB_FP64)
    h.set_engine(nat.ENGINE_PAIRS, 0, 0)
    with pytest.raises(nat.SvbError) as e:
        h.set_circuit(G.to_array([G.SRN(0)]))
    assert e.value.status == nat.SVB_ERR_UNSUPPORTED
    h11 = nat.Handle(11, 0, nat.SVB_FP64)
    h11.set_engine(nat.ENGINE_PAIRS, 0, 0)
    with pytest.raises(nat.SvbError):
        h11.set_circuit(G.to_array([G.H(0)]))
    h32 = nat.Handle(12, 0, nat.SVB_FP32)
    with pytest.raises(nat.SvbError):
        h32.set_engine(nat.ENGINE_PAIRS, 0, 0)
