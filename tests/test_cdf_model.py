"""CPU checks of the exact-CDF scheme the measurement kernels use (csrc/measure.cu),
through its numpy restatement tests/cdf_model.py: block starts equal the reference's
sequential prefix bit for bit, and samples equal the reference rule's for uniforms on
and next to every kind of boundary, on states built to hit ties, binade crossings,
zero runs, subnormal probabilities and unnormalised totals."""
import numpy as np
import pytest

import cdf_model as M


def seq_scan(re, im):
    return np.concatenate([[0.0], np.cumsum(M.probs(re, im))])


def states(n, rng):
    a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    a /= np.linalg.norm(a)
    yield "random", a.real.copy(), a.imag.copy()
    base = 2.0 ** (27 - n // 2)
    k = rng.integers(int(0.9 * base), int(1.3 * base), size=1 << n) | 1
    yield "ties", k.astype(np.float64) * 2.0 ** -27, np.zeros(1 << n)
    z = np.zeros(1 << n)
    z[(1 << (n - 1)) + 3] = 0.6
    zi = np.zeros(1 << n)
    zi[-1] = 0.8
    yield "zero_prefix", z, zi
    t = rng.random(1 << n) * 1e-160
    t[(1 << n) // 3] = 1.0
    yield "tiny_then_large", t, np.zeros(1 << n)
    yield "unnormalised", rng.random(1 << n) * 50.0, rng.random(1 << n)
    yield "plus", np.full(1 << n, 2.0 ** (-n / 2)), np.zeros(1 << n)


@pytest.mark.parametrize("n", [9, 13])
def test_block_starts_and_samples_are_the_sequential_ones(n):
    rng = np.random.default_rng(n)
    for name, re, im in states(n, rng):
        scan = seq_scan(re, im)
        T, _ = M.block_starts(M.probs(re, im))
        nb = T.size - 1
        at = np.minimum(np.arange(nb + 1) * M.BLOCK, scan.size - 1)
        assert np.array_equal(T, scan[at]), name
        js = rng.choice(scan.size - 1, size=min(60, scan.size - 1), replace=False)
        u = np.concatenate([scan[js], np.nextafter(scan[js], -np.inf), np.nextafter(scan[js], np.inf),
                            [scan[-1], np.nextafter(scan[-1], -np.inf), 1.0, 0.0, np.nan, -1.0],
                            rng.random(40)])
        assert np.array_equal(M.sample(re, im, u), M.reference_samples(re, im, u)), name


def test_grid_units_rounding():
    """round(p / 2^(e-52)) with ties flagged, against exact rational arithmetic."""
    from fractions import Fraction
    rng = np.random.default_rng(5)
    p = np.concatenate([rng.random(2000) * 2.0 ** rng.integers(-60, 0, 2000),
                        [0.0, 5e-324, 2.0 ** -1022, 0.5, 0.75, 1.0]])
    for e in (-1, -3, -20, -52):
        d, ok = M.grid_units(p, e)
        for x, di, oki in zip(p, d, ok):
            q = Fraction(float(x)) / Fraction(2) ** (e - 52)
            fl = q.numerator // q.denominator
            fr = q - fl
            if q >= 2 ** 52:
                assert not oki
                continue
            assert oki == (fr != Fraction(1, 2))
            if oki:
                assert int(di) == fl + (1 if fr > Fraction(1, 2) else 0)
