"""Generates tests/golden/matching_n30.npz: the headline circuit (n = 30, depth 40,
random-matching CX layers, seed 2024) run by the REFERENCE ITSELF.

The state comes from the reference's OpenMP CPU backend (svsim/src/svsim_cpu_omp.hpp
:196-596) built with a 64-bit IdxType by oracle/Makefile (libref_cpu_omp64.so; the
shipped 32-bit IdxType overflows at n = 29), driven through its public Simulation API
by oracle/ref_glue.cpp.  Its own measure() (:359-383) draws the first SHOTS_REF samples
with rand() seeded by SAMPLE_SEED.  The 16 GiB state cannot be committed, so the
fixture keeps what a test on the GPU can compare without it:

  * ``idx`` / ``re_at`` / ``im_at``: 4,096 amplitudes at seeded indices (plus the
    first and last index);
  * ``norm``: sum |a|^2, and ``checksum``: sum a_i w_i with w_i = cos(0.7 i) + i sin(1.3 i)
    (the weights of brickwork.npz);
  * ``sketch``: SKETCH_ROWS random-sign projections c_k = sum_i s_k(i) a_i with
    s_k(i) = r_k[i >> 15] * c_k[i & 0x7fff] and r_k, c_k = +-1 from
    numpy.random.default_rng(SKETCH_SEED) (see ``sketch_signs``).  For the error
    vector e = a_gpu - a_ref, E|c_k(e)|^2 = ||e||^2 for every k, so the mean of
    |c_k(a_gpu) - c_k(a_ref)|^2 over k estimates ||e||^2, which bounds 1 - F from above;
  * ``uniforms`` / ``samples``: the reference's own measure() samples for the first
    SHOTS_REF draws of rand() after srand(SAMPLE_SEED), and the samples of the
    reference's rule (the j with S_j <= r < S_{j+1}, else 0, S the sequential FP64
    prefix of :362-365) for SHOTS draws in all, checked equal to the reference's own
    on the first SHOTS_REF;
  * ``sample_lo`` / ``sample_hi``: the reference's S_j and S_{j+1} around each draw,
    so that a test can tell a draw within rounding distance of a CDF boundary (where a
    state that differs from the reference's in its last bits may pick a neighbour) from
    a sampling error.

Run in a container that has the reference tree (about 15 minutes on 8 cores and
~40 GiB of host memory):  python tests/golden/make_golden_n30.py
The raw reference state is cached under $SVSIM_GOLDEN_CACHE (default /tmp) so that
the fixture can be regenerated without re-running the circuit.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "sv-sim_b200"))
sys.path.insert(0, ROOT)

from svsim_b200 import circuits  # noqa: E402
from oracle.oracle import RefBackend, libc_uniforms, build  # noqa: E402

N, DEPTH, SEED = 30, 40, 2024
SAMPLE_SEED = 3030
SHOTS_REF = 48
SHOTS = 4096
SKETCH_ROWS = 64
SKETCH_SEED = 99
HALF = 15


def sketch_signs(rows: int = SKETCH_ROWS, seed: int = SKETCH_SEED):
    """(r, c): two [rows, 2^15] float64 arrays of +-1 with s_k(i) = r[k, i >> 15] * c[k, i & 0x7fff]."""
    rng = np.random.default_rng(seed)
    r = rng.integers(0, 2, size=(rows, 1 << HALF)).astype(np.float64) * 2.0 - 1.0
    c = rng.integers(0, 2, size=(rows, 1 << HALF)).astype(np.float64) * 2.0 - 1.0
    return r, c


def sketch(re: np.ndarray, im: np.ndarray) -> np.ndarray:
    """c_k = sum_i s_k(i) (re_i + i im_i) for a 2^30 state."""
    r, c = sketch_signs()
    a_re = re.reshape(1 << HALF, 1 << HALF) @ c.T          # [hi, k]
    a_im = im.reshape(1 << HALF, 1 << HALF) @ c.T
    return np.einsum("kh,hk->k", r, a_re) + 1j * np.einsum("kh,hk->k", r, a_im)


def checksum(re: np.ndarray, im: np.ndarray, chunk: int = 1 << 24) -> complex:
    tot = 0j
    for s in range(0, re.size, chunk):
        i = np.arange(s, min(s + chunk, re.size), dtype=np.float64)
        w = np.cos(0.7 * i) + 1j * np.sin(1.3 * i)
        tot += np.sum((re[s:s + chunk] + 1j * im[s:s + chunk]) * w)
    return tot


def reference_rule(scan: np.ndarray, r: np.ndarray) -> np.ndarray:
    """The j with S_j <= r < S_{j+1}, else 0 (svsim_cpu_omp.hpp:372-375), for a
    non-decreasing S of 2^n + 1 entries."""
    dim = scan.size - 1
    k = np.searchsorted(scan, r, side="right") - 1      # largest k with S_k <= r
    return np.where((k >= 0) & (k < dim), k, 0).astype(np.uint64)


def main():
    cache = os.environ.get("SVSIM_GOLDEN_CACHE", "/tmp")
    raw = os.path.join(cache, f"svsim_ref_matching_n{N}_d{DEPTH}_s{SEED}.npz")
    gates = circuits.random_matching_circuit(N, DEPTH, seed=SEED)
    if os.path.exists(raw):
        z = np.load(raw)
        re, im, ref_samples = z["re"], z["im"], z["samples"]
        sim_s = float(z["sim_s"])
    else:
        build(reference=True)
        ref = RefBackend("omp64")
        t0 = time.time()
        r = ref.simulate(N, gates, threads=os.cpu_count(), shots=SHOTS_REF, seed=SAMPLE_SEED)
        sim_s = r["sim_ms"] / 1e3
        print(f"reference cpu_omp64 n={N}: sim {sim_s:.1f} s, total {time.time() - t0:.1f} s",
              flush=True)
        re, im, ref_samples = r["re"], r["im"], r["samples"]
        np.savez(raw, re=re, im=im, samples=ref_samples, sim_s=sim_s)

    rng = np.random.default_rng(77)
    idx = np.unique(np.concatenate([[0, (1 << N) - 1],
                                    rng.choice(1 << N, size=4096, replace=False)])).astype(np.uint64)
    sk = sketch(re, im)
    cs = checksum(re, im)

    # the reference's sequential prefix (svsim_cpu_omp.hpp:362-365): p_i = re*re + im*im
    # without contraction, S_0 = 0, S_{i+1} = S_i + p_i in index order
    scan = np.empty((1 << N) + 1)
    scan[0] = 0.0
    p = re * re
    p += im * im
    np.cumsum(p, out=scan[1:])
    norm = float(scan[-1])
    del p

    u = libc_uniforms(SAMPLE_SEED, SHOTS)
    samples = reference_rule(scan, u)
    if not np.array_equal(samples[:SHOTS_REF], ref_samples):
        raise SystemExit("the restated rule disagrees with the reference's measure()")

    # the reference's CDF interval [S_j, S_{j+1}) of every sample: a state that differs
    # from the reference's by rounding moves S by far less than the distance of most
    # draws to these ends, and a test can tell such a draw from a sampling error
    s_lo = scan[samples.astype(np.int64)]
    s_hi = scan[samples.astype(np.int64) + 1]
    out = os.path.join(HERE, f"matching_n{N}.npz")
    np.savez_compressed(
        out, n=np.array([N]), depth=np.array([DEPTH]), seed=np.array([SEED]), gates=gates,
        idx=idx, re_at=re[idx], im_at=im[idx], norm=np.array([norm]),
        checksum=np.array([cs]), sketch=sk, sketch_rows=np.array([SKETCH_ROWS]),
        sketch_seed=np.array([SKETCH_SEED]), sample_seed=np.array([SAMPLE_SEED]),
        uniforms=u, samples=samples, shots_ref=np.array([SHOTS_REF]),
        sample_lo=s_lo, sample_hi=s_hi,
        ref_sim_seconds=np.array([sim_s]), ref_threads=np.array([os.cpu_count()]))
    print(out, os.path.getsize(out), "norm", norm, "checksum", cs)


if __name__ == "__main__":
    main()
