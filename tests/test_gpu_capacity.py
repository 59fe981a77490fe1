"""Capacity: the largest states one B200 holds, n=33 FP64 (staged, 128 GiB) and n=34 FP32
(fused tensor-core, 128 GiB), on depth-20 random-matching circuits.  No CPU checker
reaches these sizes, so the checks are size-independent: the FP64 CDF total is 1,
4096 samples fall inside the state and are spread out, and the inverse circuit brings
the state back to |0..0> (every <Z_q> = 1, every sample 0)."""
import numpy as np
import pytest

from svsim_b200 import circuits

pytestmark = pytest.mark.gpu

SHOTS = 4096


def z_terms(n):
    from svsim_b200.gates import PAULI_DTYPE
    t = np.zeros(n, dtype=PAULI_DTYPE)
    for q in range(n):
        t[q] = (1.0 / n, 0, 1 << q)
    return t


@pytest.mark.parametrize("n,prec,engine,k,tol", [
    (33, "fp64", "staged", 0, 1e-10),
    (33, "fp64", "pairs", 0, 1e-10),
    (34, "fp32", "fused", 5, 2e-4),
])
def test_round_trip_and_sampling(n, prec, engine, k, tol):
    from svsim_b200 import _native as nat
    P = nat.SVB_FP64 if prec == "fp64" else nat.SVB_FP32
    E = {"staged": nat.ENGINE_STAGED, "pairs": nat.ENGINE_PAIRS, "fused": nat.ENGINE_FUSED}[engine]
    circ = circuits.random_matching_circuit(n, 20, seed=2024)
    h = nat.Handle(n, 0, P)
    try:
        h.set_engine(E, 0, k)
        h.set_circuit(circ)
        h.run()
        h.sync()
        uni = np.random.default_rng(5).random(SHOTS)
        samples, total = h.measure(uni)
        assert abs(total - 1.0) <= tol
        assert np.all(samples < (1 << n))
        assert len(np.unique(samples)) >= SHOTS - 8          # a 2^n-outcome random state
        # below the CDF total the sample order follows the uniforms (larger uniform, larger
        # or equal index); at or above it the reference's rule returns 0 (an FP32 state's
        # norm sits a little below 1)
        inside = uni < total
        order = np.argsort(uni[inside])
        assert np.all(np.diff(samples[inside][order].astype(np.int64)) >= 0)
        assert np.count_nonzero(samples[~inside]) == 0
        h.set_circuit(circuits.inverse_circuit(circ))
        h.run()
        h.sync()
        assert h.expectation(z_terms(n)) >= 1.0 - tol
        back, total2 = h.measure(uni)
        assert abs(total2 - 1.0) <= tol
        assert np.count_nonzero(back) == 0
    finally:
        h.close()
