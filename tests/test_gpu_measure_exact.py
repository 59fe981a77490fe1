"""Sampling is the reference's, bit for bit, at the edges of its rule.

The reference draws r and keeps the j with S_j <= r < S_{j+1}, where S is its
sequential FP64 prefix of |a|^2 (svsim_nvgpu_sin.cuh:359-383).  A prefix summed in
any other order can put a boundary one ulp away and so change the sample of an r that
lies on or next to some S_j.  These tests place uniforms exactly on the reference's own
S_j (computed from the GPU's state by the C oracle's sequential scan, which is pinned to
the reference) and on both neighbouring doubles, on adversarial states built to hit
every path of the GPU's exact prefix: binade crossings, ties (p/u with a fraction of
exactly one half, where round-half-even depends on the running sum), long runs of zero
probability, tiny probabilities before a large one, unnormalised and FP32 states."""
import numpy as np
import pytest

from svsim_b200 import circuits

pytestmark = pytest.mark.gpu


def native():
    from svsim_b200 import _native
    return _native


def sequential_scan(re, im):
    p = re * re
    p += im * im
    scan = np.empty(p.size + 1)
    scan[0] = 0.0
    np.cumsum(p, out=scan[1:])          # add.accumulate: index order, like the reference
    return scan


def edge_uniforms(scan, rng, count=300):
    js = rng.choice(scan.size - 1, size=min(count, scan.size - 1), replace=False)
    sj = scan[js]
    tail = [scan[-1], np.nextafter(scan[-1], -np.inf), np.nextafter(scan[-1], np.inf), 1.0,
            np.nextafter(1.0, -np.inf), 0.0, -0.0, np.nextafter(0.0, 1.0), -1e-300, np.nan]
    return np.concatenate([sj, np.nextafter(sj, -np.inf), np.nextafter(sj, np.inf), tail,
                           rng.random(512)])


def check_state(oracle, h, n, rng, count=300):
    re, im = h.get_state()
    scan = sequential_scan(re, im)
    u = edge_uniforms(scan, rng, count)
    got, total = h.measure(u)
    want, wtotal = oracle.measure(n, re, im, u)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, [(float(u[i]), int(got[i]), int(want[i])) for i in bad[:8]]
    assert total == wtotal == scan[-1]          # bit-identical total
    return got


@pytest.mark.parametrize("n,engine", [(16, 0), (16, 1), (21, 0), (21, 2)])
def test_edges_on_random_circuit_states(oracle, n, engine):
    nat = native()
    h = nat.Handle(n, 0, nat.SVB_FP64)
    h.set_engine(engine, 0, 0)
    h.set_circuit(circuits.random_matching_circuit(n, 6, seed=100 + n))
    h.run()
    h.sync()
    check_state(oracle, h, n, np.random.default_rng(n))


def tie_state(n, rng):
    """re_i = k_i 2^-27 with k_i odd: p_i = k_i^2 2^-54 exactly, an odd multiple of 2^-54.
    While 1/2 <= S < 1 the grid unit is 2^-53, so every p_i/u has a fraction of exactly
    1/2.  The k_i are sized for a total of about 1.2."""
    base = 2.0 ** (27 - n // 2)
    k = rng.integers(int(0.9 * base), int(1.3 * base), size=1 << n) | 1
    return k.astype(np.float64) * 2.0 ** -27, np.zeros(1 << n)


def zero_prefix_state(n, rng):
    re = np.zeros(1 << n)
    im = np.zeros(1 << n)
    re[(1 << (n - 1)) + 3] = 0.6
    im[(1 << (n - 1)) + 4097] = 0.8
    im[-1] = 1e-3
    return re, im


def tiny_then_large_state(n, rng):
    re = rng.random(1 << n) * 1e-160        # p ~ 1e-320: subnormal probabilities first
    re[(1 << n) // 3] = 1.0
    im = np.zeros(1 << n)
    im[(1 << n) // 3 + 1:] = rng.random((1 << n) - (1 << n) // 3 - 1) * 2.0 ** -20
    return re, im


def sparse_state(n, rng):
    a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    a[rng.random(1 << n) < 0.97] = 0.0       # exact zeros between the non-zero amplitudes
    a /= np.linalg.norm(a)
    return a.real.copy(), a.imag.copy()


def unnormalised_state(n, rng):
    return rng.random(1 << n) * 50.0, rng.random(1 << n)


def plus_state(n, rng):
    return np.full(1 << n, 2.0 ** (-n / 2)), np.zeros(1 << n)


@pytest.mark.parametrize("maker", [tie_state, zero_prefix_state, tiny_then_large_state,
                                   sparse_state, unnormalised_state, plus_state])
@pytest.mark.parametrize("n", [14, 20])
def test_edges_on_adversarial_states(oracle, maker, n):
    nat = native()
    rng = np.random.default_rng(sum(map(ord, maker.__name__)) + n)
    re, im = maker(n, rng)
    h = nat.Handle(n, 0, nat.SVB_FP64)
    h.set_state(re, im)
    check_state(oracle, h, n, rng)


def test_tie_state_really_ties():
    """The tie state puts exact halves on the grid of the top binade (sanity of the test)."""
    rng = np.random.default_rng(3)
    re, im = tie_state(20, rng)
    scan = sequential_scan(re, im)
    assert scan[-1] > 1.0
    top = (scan[:-1] >= 0.5) & (scan[:-1] < 1.0)       # S before adding p_i
    assert top.sum() > 100000
    p = re * re
    frac = (p[top] / 2.0 ** -53) % 1.0
    assert np.all(frac == 0.5)


@pytest.mark.parametrize("n", [13, 22])
def test_edges_on_fp32_states(oracle, n):
    """FP32 amplitudes are widened to FP64 and sampled with the same rule."""
    nat = native()
    h = nat.Handle(n, 0, nat.SVB_FP32)
    h.set_circuit(circuits.random_matching_circuit(n, 4, seed=n))
    h.run()
    h.sync()
    check_state(oracle, h, n, np.random.default_rng(7 * n))


def test_small_states(oracle):
    nat = native()
    for n in (1, 2, 3, 5, 11, 12):
        h = nat.Handle(n, 0, nat.SVB_FP64)
        h.set_circuit(circuits.random_matching_circuit(n, 3, seed=n))
        h.run()
        h.sync()
        check_state(oracle, h, n, np.random.default_rng(n), count=min(300, 1 << n))
