"""The fused tensor-core FP32 engine (tcgen05, split TF32) against the FP64 oracle:
1-F <= 1e-6 and the largest amplitude error reported."""
import numpy as np
import pytest

from conftest import fidelity
from svsim_b200 import circuits, gates as G

pytestmark = pytest.mark.gpu


def run_fused(n, gates, k):
    from svsim_b200 import _native as nat
    h = nat.Handle(n, 0, nat.SVB_FP32)
    h.set_engine(nat.ENGINE_FUSED, 0, k)
    h.set_circuit(gates)
    h.run()
    h.sync()
    return h


@pytest.mark.parametrize("k", [3, 4, 5, 6])
@pytest.mark.parametrize("n", [12, 14, 17, 22])
def test_fused_matches_oracle(oracle, n, k):
    """n = 12..17 give each CTA one tile; n = 22 (1,024 tiles) gives each several, so both
    tile slots (three at k = 6), the prefetch buffers' reuse and the output stage's reuse
    run."""
    g = circuits.random_matching_circuit(n, 8, seed=100 * n + k)
    h = run_fused(n, g, k)
    re, im = h.get_state()
    ore, oim = oracle.run(n, g)
    infid = 1 - fidelity(re + 1j * im, ore + 1j * oim)
    assert infid <= 1e-6, infid
    assert np.max(np.abs((re + 1j * im) - (ore + 1j * oim))) <= 1e-5


def test_fused_every_op(oracle):
    import math
    n = 13
    rng = np.random.default_rng(3)
    gl = G.from_array(circuits.random_matching_circuit(n, 1, seed=3))
    for _ in range(3):
        for name in G.OP_NAMES:
            if name == "SRN":
                continue
            qs = [int(x) for x in rng.permutation(n)[:G.N_QUBITS[name]]]
            npar = {"U3": 3, "U2": 2, "CU3": 3}.get(name, 1 if name in (
                "U1", "RX", "RY", "RZ", "CRX", "CRY", "CRZ", "CU1", "RXX", "RZZ", "RYY", "R") else 0)
            gl.append(G.FACTORIES[name](*([rng.uniform(-math.pi, math.pi) for _ in range(npar)] + qs)))
    g = G.to_array(gl)
    ore, oim = oracle.run(n, g)
    for k in (4, 6):
        h = run_fused(n, g, k)
        re, im = h.get_state()
        assert 1 - fidelity(re + 1j * im, ore + 1j * oim) <= 1e-6, k


@pytest.mark.parametrize("k", [4, 5, 6])
def test_fused_vs_fp64_on_device(k):
    from svsim_b200 import _native as nat
    n = 22
    g = circuits.random_matching_circuit(n, 10, seed=5)
    h32 = run_fused(n, g, k)
    h64 = nat.Handle(n, 0, nat.SVB_FP64)
    h64.set_circuit(g)
    h64.run()
    f, d = h64.compare(h32)
    assert 1 - f <= 1e-6 and d <= 1e-5


def test_fused_rejects_srn_and_fp64():
    from svsim_b200 import _native as nat
    h = nat.Handle(12, 0, nat.SVB_FP32)
    for k in (4, 6):
        h.set_engine(nat.ENGINE_FUSED, 0, k)
        with pytest.raises(nat.SvbError) as e:
            h.set_circuit(G.to_array([G.SRN(0)]))
        assert e.value.status == nat.SVB_ERR_UNSUPPORTED
    with pytest.raises(nat.SvbError):
        h.set_engine(nat.ENGINE_FUSED, 0, 7)
    h64 = nat.Handle(12, 0, nat.SVB_FP64)
    with pytest.raises(nat.SvbError):
        h64.set_engine(nat.ENGINE_FUSED, 0, 4)


def test_fused_run_keeps_unit_norm_and_small_amplitude_error():
    """The tensor cores truncate their FP32 sums, so without the closing FP64
    renormalisation the norm of a deep fused run decays by ~1e-7 per gate; with it the
    norm stays 1 to FP32 rounding and the largest amplitude error stays at FP32 level."""
    from svsim_b200 import _native as nat
    n = 20
    g = circuits.random_matching_circuit(n, 40, seed=9)
    h64 = nat.Handle(n, 0, nat.SVB_FP64)
    h64.set_circuit(g)
    h64.run()
    amp = 2.0 ** (-n / 2)
    for k in (4, 6):
        h32 = run_fused(n, g, k)
        assert abs(h32.norm2() - 1.0) <= 2e-6
        f, d = h64.compare(h32)
        assert 1 - f <= 1e-9 and d <= 2e-4 * amp, (k, 1 - f, d)


def test_auto_engine_runs_fp32_circuits_on_the_fused_engine(oracle):
    """AUTO sends FP32 circuits of >= 12 qubits to the fused engine, and those with SRN
    (not complex-linear) to the staged engine; both match the oracle."""
    from svsim_b200 import _native as nat
    n = 14
    g = circuits.random_matching_circuit(n, 6, seed=21)
    h = nat.Handle(n, 0, nat.SVB_FP32)
    h.set_circuit(g)
    assert h.plan_info().engine == nat.ENGINE_FUSED
    h.run()
    re, im = h.get_state()
    ore, oim = oracle.run(n, g)
    assert 1 - fidelity(re + 1j * im, ore + 1j * oim) <= 1e-6
    g2 = G.to_array(G.from_array(g) + [G.SRN(3)])
    h.set_circuit(g2)
    assert h.plan_info().engine == nat.ENGINE_STAGED
