"""Host logic of the staged engine: plans executed on the CPU by tests/native's emulator
(the tile kernel's own index helpers) must reproduce the oracle."""
import ctypes
import math

import numpy as np
import pytest

from conftest import cx_dense_circuit, fidelity
from svsim_b200 import circuits, gates as G

_dp = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def emu():
    import build_emulator
    lib = ctypes.CDLL(build_emulator.build())
    return lib


def run_emu(lib, n, gates, M, precision=0, state=None):
    if state is None:
        re = np.zeros(1 << n)
        im = np.zeros(1 << n)
        re[0] = 1.0
    else:
        re, im = state[0].copy(), state[1].copy()
    np_, ns = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib.emu_staged_run(n, gates.ctypes.data, ctypes.c_size_t(len(gates)), M, precision,
                            re.ctypes.data_as(_dp), im.ctypes.data_as(_dp), ctypes.byref(np_),
                            ctypes.byref(ns))
    assert rc == 0, f"emulator rc {rc}"
    return re, im, np_.value


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


@pytest.mark.parametrize("n,M", [(10, 10), (12, 10), (12, 11), (12, 12), (13, 12), (15, 12)])
def test_staged_plan_random_matching_fp64(emu, oracle, n, M):
    g = circuits.random_matching_circuit(n, 10, seed=n * 31 + M)
    re, im, passes = run_emu(emu, n, g, M)
    ore, oim = oracle.run(n, g)
    assert np.max(np.abs(re - ore)) < 1e-13 and np.max(np.abs(im - oim)) < 1e-13
    assert passes < len(g)


@pytest.mark.parametrize("M", [10, 11, 12])
def test_staged_plan_every_op_fp64(emu, oracle, M):
    """All 38 ops, including the non-unitary SRN and R, interleaved at random."""
    n = 12
    g = mixed_circuit(n, 4, seed=M)
    re, im, _ = run_emu(emu, n, g, M)
    ore, oim = oracle.run(n, g)
    assert np.max(np.abs(re - ore)) < 1e-12 and np.max(np.abs(im - oim)) < 1e-12


@pytest.mark.parametrize("M", [11, 12, 13])
def test_staged_plan_every_op_fp32(emu, oracle, M):
    n = 13
    g = mixed_circuit(n, 3, seed=100 + M)
    re, im, _ = run_emu(emu, n, g, M, precision=1)
    ore, oim = oracle.run(n, g)
    assert 1 - fidelity(re + 1j * im, ore + 1j * oim) < 1e-6


def test_staged_plan_from_arbitrary_state(emu, oracle):
    n = 11
    rng = np.random.default_rng(5)
    st = (rng.standard_normal(1 << n), rng.standard_normal(1 << n))
    g = mixed_circuit(n, 2, seed=9)
    re, im, _ = run_emu(emu, n, g, 11, state=st)
    ore, oim = oracle.run(n, g, state=st)
    assert np.max(np.abs(re - ore)) < 1e-11 and np.max(np.abs(im - oim)) < 1e-11


def test_srn_is_ordered_against_complex_gates(emu, oracle):
    """SRN (svsim_nvgpu_sin.cuh:894-907) is only real-linear: moving it past a complex
    gate on another qubit changes the result, so the plan must not reorder it."""
    g = G.to_array([G.H(2), G.SRN(0), G.W(5), G.U2(-0.68, 0.36, 2)])
    re, im, _ = run_emu(emu, 12, g, 12)
    ore, oim = oracle.run(12, g)
    assert np.max(np.abs(re - ore)) < 1e-14 and np.max(np.abs(im - oim)) < 1e-14


def test_plan_pass_counts_headline_circuit(emu):
    """The n=30 depth-40 circuit (1,800 gates) needs far fewer passes than sweeps."""
    g = circuits.random_matching_circuit(30, 40)
    a, b, c, d = (ctypes.c_uint64() for _ in range(4))
    rc = emu.emu_plan_stats(30, g.ctypes.data, ctypes.c_size_t(len(g)), 12, 0, ctypes.byref(a),
                            ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))
    assert rc == 0
    assert d.value == 1800
    assert a.value <= 80          # passes (each one read + one write of the state)


def run_fused_emu(lib, n, gates, k):
    re = np.zeros(1 << n)
    im = np.zeros(1 << n)
    re[0] = 1.0
    a, b = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib.emu_fused_run(n, gates.ctypes.data, ctypes.c_size_t(len(gates)), k,
                           re.ctypes.data_as(_dp), im.ctypes.data_as(_dp), ctypes.byref(a),
                           ctypes.byref(b))
    return rc, re, im, a.value, b.value


@pytest.mark.parametrize("n,k", [(12, 5), (13, 4), (14, 3), (15, 5)])
def test_fused_plan_random_matching(emu, oracle, n, k):
    """Fusion into k-qubit blocks, operand layouts and index tables of the tensor-core
    engine, executed on the CPU (MMA in FP64): only the FP32 rounding of the gates remains."""
    g = circuits.random_matching_circuit(n, 6, seed=n * 7 + k)
    rc, re, im, passes, blocks = run_fused_emu(emu, n, g, k)
    assert rc == 0
    ore, oim = oracle.run(n, g)
    assert 1 - fidelity(re + 1j * im, ore + 1j * oim) < 1e-12
    assert np.max(np.abs(re - ore)) < 1e-7 and blocks < len(g)


def test_fused_plan_every_op_but_srn(emu, oracle):
    n = 12
    g = mixed_circuit(n, 3, seed=21)
    g = g[g["op"] != G.OP["SRN"]]
    rc, re, im, _, _ = run_fused_emu(emu, n, g, 4)
    assert rc == 0
    ore, oim = oracle.run(n, g)
    assert 1 - fidelity(re + 1j * im, ore + 1j * oim) < 1e-12


def test_fused_plan_rejects_srn(emu):
    g = G.to_array([G.H(0), G.SRN(3)])
    rc, *_ = run_fused_emu(emu, 12, g, 4)
    assert rc == -3


def run_fused6_emu(lib, n, gates):
    re = np.zeros(1 << n)
    im = np.zeros(1 << n)
    re[0] = 1.0
    a = ctypes.c_uint64()
    rc = lib.emu_fused6_run(n, gates.ctypes.data, ctypes.c_size_t(len(gates)), re.ctypes.data_as(_dp),
                            im.ctypes.data_as(_dp), ctypes.byref(a))
    return rc, re, im, a.value


@pytest.mark.parametrize("n,depth", [(12, 6), (13, 5), (15, 4), (16, 3)])
def test_fused6_plan_random_matching(emu, oracle, n, depth):
    """Fusion width 6: greedy 6-qubit blocks (one per pass), the B-operand plane offsets,
    the canonical K-major reads of the MMA and the output offsets, executed on the CPU
    (MMA in FP64): only the TF32 hi + lo rounding of the gate remains."""
    g = circuits.random_matching_circuit(n, depth, seed=n * 11 + depth)
    rc, re, im, passes = run_fused6_emu(emu, n, g)
    assert rc == 0
    ore, oim = oracle.run(n, g)
    assert 1 - fidelity(re + 1j * im, ore + 1j * oim) < 1e-12
    assert np.max(np.abs(re - ore)) < 1e-7 and passes < len(g)


def test_fused6_plan_every_op_but_srn(emu, oracle):
    n = 13
    g = mixed_circuit(n, 3, seed=33)
    g = g[g["op"] != G.OP["SRN"]]
    rc, re, im, _ = run_fused6_emu(emu, n, g)
    assert rc == 0
    ore, oim = oracle.run(n, g)
    assert 1 - fidelity(re + 1j * im, ore + 1j * oim) < 1e-12


def test_fused6_plan_low_qubit_targets(emu, oracle):
    """Blocks whose targets include qubits 0 and 1 (both targets: the 2-way-conflict
    layout), only qubit 0, or neither, and blocks padded to 6 targets."""
    gl = []
    for q in range(12):
        gl.append(G.U3(0.3 + 0.1 * q, 0.2 * q, -0.4, q))
    gl += [G.CX(0, 1), G.CX(1, 5), G.CX(0, 7), G.U3(0.5, 0.1, 0.2, 0), G.CX(2, 3), G.CX(9, 11),
           G.CX(4, 13), G.H(12), G.CX(12, 0), G.RZ(0.7, 1), G.CX(10, 2)]
    g = G.to_array(gl)
    rc, re, im, _ = run_fused6_emu(emu, 14, g)
    assert rc == 0
    ore, oim = oracle.run(14, g)
    assert 1 - fidelity(re + 1j * im, ore + 1j * oim) < 1e-12


def test_fused6_plan_headline_circuit_blocks(emu):
    """n = 30, depth 40: 1,800 gates in at most 150 six-qubit blocks (passes), and at
    most 190 five-qubit blocks in 70 passes."""
    g = circuits.random_matching_circuit(30, 40, seed=2024)
    a, b = ctypes.c_uint64(), ctypes.c_uint64()
    rc = emu.emu_fused_stats(30, g.ctypes.data, ctypes.c_size_t(len(g)), 6, ctypes.byref(a), ctypes.byref(b))
    assert rc == 0
    assert a.value == b.value and a.value <= 150
    rc = emu.emu_fused_stats(30, g.ctypes.data, ctypes.c_size_t(len(g)), 5, ctypes.byref(a), ctypes.byref(b))
    assert rc == 0 and a.value <= 70 and b.value <= 190


def run_pairs_emu(lib, n, gates):
    re = np.zeros(1 << n)
    im = np.zeros(1 << n)
    st = np.zeros(4, dtype=np.uint64)
    vp = ctypes.c_void_p
    rc = lib.emu_pairs_run(ctypes.c_uint32(n), vp(gates.ctypes.data), ctypes.c_size_t(len(gates)),
                           vp(re.ctypes.data), vp(im.ctypes.data), vp(st.ctypes.data))
    return rc, re, im, st


@pytest.mark.parametrize("n,depth", [(12, 6), (13, 8), (16, 10), (17, 6)])
def test_pair_plan_random_matching(emu, oracle, n, depth):
    """Pair-engine plan (two-qubit blocks, lane/register exchanges, relayouts, tile-
    selected variants) run thread by thread with the kernel's data movement and MMA
    fragment rules, against the oracle."""
    g = circuits.random_matching_circuit(n, depth, seed=n + depth)
    rc, re, im, st = run_pairs_emu(emu, n, g)
    assert rc == 0, rc
    ore, oim = oracle.run(n, g)
    assert np.max(np.abs((re + 1j * im) - (ore + 1j * oim))) < 1e-13
    assert st[1] <= len(g)                  # no more blocks than gates


def test_pair_plan_every_op_but_srn_and_qaoa(emu, oracle):
    for n, g in [(15, mixed_circuit(15, 3, seed=31)),
                 (14, circuits.qaoa_instances(1, n_min=14, n_max=14, seed=5)[0].circuit()),
                 (16, circuits.brickwork_circuit(16, 20))]:
        g = g[g["op"] != G.OP["SRN"]]
        rc, re, im, _ = run_pairs_emu(emu, n, g)
        assert rc == 0, rc
        ore, oim = oracle.run(n, g)
        assert np.max(np.abs((re + 1j * im) - (ore + 1j * oim))) < 1e-13


def test_pair_plan_rejects_srn_and_small_states(emu):
    g = G.to_array([G.H(0), G.SRN(1)])
    assert run_pairs_emu(emu, 12, g)[0] == -6
    assert run_pairs_emu(emu, 11, G.to_array([G.H(0)]))[0] == -6


def test_pair_plan_shared_memory_staging(emu):
    """Every pass's ops and layouts, and its gate fragments where they fit, are copied
    into shared memory beside the 64 KiB tile: the largest copy stays within two CTAs per
    SM, the n=30 headline circuit stages every pass, and the CX-dense n=12 circuit (run on
    the GPU by test_pair_engine_pass_with_gates_beyond_shared_memory) has passes whose
    gates stay in global memory."""
    def stats(n, depth):
        g = circuits.random_matching_circuit(n, depth, seed=1)
        st = np.zeros(8, dtype=np.uint64)
        rc = emu.emu_pairs_stats(ctypes.c_uint32(n), ctypes.c_void_p(g.ctypes.data), ctypes.c_size_t(len(g)),
                                 ctypes.c_void_p(st.ctypes.data))
        assert rc == 0
        return st
    tile = 16 << 12
    for n, depth in ((12, 60), (20, 40), (30, 40)):
        st = stats(n, depth)
        assert tile + int(st[5]) <= 112 * 1024
    assert stats(30, 40)[4] == 0
    g = cx_dense_circuit()
    st = np.zeros(8, dtype=np.uint64)
    assert emu.emu_pairs_stats(ctypes.c_uint32(12), ctypes.c_void_p(g.ctypes.data), ctypes.c_size_t(len(g)),
                               ctypes.c_void_p(st.ctypes.data)) == 0
    assert st[4] >= 1 and tile + int(st[5]) <= 112 * 1024


def test_pair_plan_cx_dense_vs_oracle(emu, oracle):
    """The CX-dense circuit (passes whose gates stay in global memory) through the pair
    plan emulator."""
    g = cx_dense_circuit()
    rc, re, im, _ = run_pairs_emu(emu, 12, g)
    assert rc == 0, rc
    ore, oim = oracle.run(12, g)
    assert np.max(np.abs((re + 1j * im) - (ore + 1j * oim))) < 1e-13


# ---- every plan on a random input state -------------------------------------------------
# From |0..0>, an op that only multiplies amplitudes with some qubit at 1 (a phase on a
# non-local qubit, a tile-selected variant) is invisible until the state spreads; a plan that
# drops one passes every test that starts there.  These run each planner on circuits heavy
# in diagonal ops, from a random normalised state, against the oracle applied to that state.

def random_state(n, seed):
    rng = np.random.default_rng(seed)
    s = rng.normal(size=(2, 1 << n))
    s /= np.sqrt((s ** 2).sum())
    return s[0].copy(), s[1].copy()


def diagonal_heavy_circuit(n, m, seed):
    rng = np.random.default_rng(seed)
    gl = []
    for _ in range(m):
        r = rng.random()
        q = int(rng.integers(n))
        q2 = int(rng.integers(n - 1))
        q2 += q2 >= q
        if r < 0.3:
            gl.append(G.RZ(rng.uniform(-3, 3), q))
        elif r < 0.4:
            gl.append(G.T(q))
        elif r < 0.5:
            gl.append(G.U1(rng.uniform(-3, 3), q))
        elif r < 0.65:
            gl.append(G.CX(q, q2))
        elif r < 0.75:
            gl.append(G.CZ(q, q2))
        elif r < 0.85:
            gl.append(G.RY(rng.uniform(-3, 3), q))
        else:
            gl.append(G.U3(*rng.uniform(-3, 3, 3), q))
    return G.to_array(gl)


def ansatz_segment(n, lo, hi):
    """Ops lo..hi of the hardware-efficient ansatz: a segment that opens with a run of RZ
    (the adjoint's forward checkpoints cut the circuit like this)."""
    pc = circuits.hardware_efficient_ansatz(n=n, layers=2, seed=7)
    return np.ascontiguousarray(pc.evaluated(pc.params)[lo:hi])


STATE_CASES = [(n, diagonal_heavy_circuit(n, m, seed)) for n, m, seed in
               ((12, 60, 1), (13, 40, 2), (14, 80, 3), (15, 50, 4), (17, 90, 5))]
# n = 18, a pass of 12 local qubits: the segment's first RZ on 5 or more non-local qubits
# fill the tile phase twice over before any block
STATE_CASES += [(18, ansatz_segment(18, 22, 46)), (18, ansatz_segment(18, 58, 82))]


@pytest.mark.parametrize("case", range(len(STATE_CASES)))
def test_pair_plan_on_random_state(emu, oracle, case):
    n, g = STATE_CASES[case]
    re, im = random_state(n, case)
    ore, oim = oracle.run(n, g, state=(re, im))
    st = np.zeros(4, dtype=np.uint64)
    vp = ctypes.c_void_p
    rc = emu.emu_pairs_run_from(ctypes.c_uint32(n), vp(g.ctypes.data), ctypes.c_size_t(len(g)),
                                vp(re.ctypes.data), vp(im.ctypes.data), vp(st.ctypes.data))
    assert rc == 0
    assert np.max(np.abs((re + 1j * im) - (ore + 1j * oim))) < 1e-13


@pytest.mark.parametrize("case", range(len(STATE_CASES)))
def test_staged_plan_on_random_state(emu, oracle, case):
    n, g = STATE_CASES[case]
    st = random_state(n, case)
    ore, oim = oracle.run(n, g, state=st)
    for M in (10, 12):
        re, im, _ = run_emu(emu, n, g, M, state=st)
        assert np.max(np.abs((re + 1j * im) - (ore + 1j * oim))) < 1e-13, M


@pytest.mark.parametrize("case", range(len(STATE_CASES)))
def test_fused_plans_on_random_state(emu, oracle, case):
    n, g = STATE_CASES[case]
    st = random_state(n, case)
    ore, oim = oracle.run(n, g, state=st)
    for k in (3, 4, 5, 6):
        re, im = st[0].copy(), st[1].copy()
        if k < 6:
            a, b = ctypes.c_uint64(), ctypes.c_uint64()
            rc = emu.emu_fused_run(n, g.ctypes.data, ctypes.c_size_t(len(g)), k, re.ctypes.data_as(_dp),
                                   im.ctypes.data_as(_dp), ctypes.byref(a), ctypes.byref(b))
        else:
            a = ctypes.c_uint64()
            rc = emu.emu_fused6_run(n, g.ctypes.data, ctypes.c_size_t(len(g)), re.ctypes.data_as(_dp),
                                    im.ctypes.data_as(_dp), ctypes.byref(a))
        assert rc == 0, k
        assert 1 - fidelity(re + 1j * im, ore + 1j * oim) < 1e-12, k


def plan_cost(st):
    """The pair planner's cost model, in block units: blocks + 0.49 exchanges + 0.36 lane
    permutations + 2.05 relayouts + 0.6 passes."""
    return int(st[1]) + 0.49 * int(st[2]) + 0.36 * int(st[6]) + 2.05 * int(st[3]) + 0.6 * int(st[0])


@pytest.mark.parametrize("n,depth,seed", [(14, 12, 1), (18, 20, 2), (20, 40, 2024), (24, 40, 2024), (30, 40, 2024)])
def test_pair_plan_keeps_the_cheaper_pass_cut(emu, n, depth, seed):
    """plan_pairs plans the program-order and the seeded pass cut and keeps the cheaper by
    the cost model: never above the program-order plan; at n = 30 the seeded one (48
    passes against 50)."""
    g = circuits.random_matching_circuit(n, depth, seed=seed)
    both, one = np.zeros(8, dtype=np.uint64), np.zeros(8, dtype=np.uint64)
    vp = ctypes.c_void_p
    assert emu.emu_pairs_stats(ctypes.c_uint32(n), vp(g.ctypes.data), ctypes.c_size_t(len(g)), vp(both.ctypes.data)) == 0
    assert emu.emu_pairs_stats_one_cut(ctypes.c_uint32(n), vp(g.ctypes.data), ctypes.c_size_t(len(g)),
                                       vp(one.ctypes.data)) == 0
    assert plan_cost(both) <= plan_cost(one) + 1e-9
    if n == 30:
        assert int(one[0]) == 50 and int(both[0]) == 48 and plan_cost(both) < plan_cost(one)
