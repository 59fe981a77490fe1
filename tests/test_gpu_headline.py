"""Parity at the headline size: the n = 30, depth-40 random-matching circuit (1,800 gates,
seed 2024) on every engine, against the reference's own OpenMP CPU backend
(svsim_cpu_omp.hpp:196-596, 64-bit IdxType build) through the golden fixture
tests/golden/matching_n30.npz (made by tests/golden/make_golden_n30.py).

The 16 GiB reference state is not in the fixture; it keeps 4,097 amplitudes, the norm, a
weighted checksum, 64 random-sign projections (a sketch: the mean of |c_k(a) - c_k(b)|^2
estimates ||a - b||^2, an upper bound of 1 - F for unit vectors) and the reference rule's
samples of 4,096 draws with their CDF intervals.  Bars: FP64 max|d amp| <= 1e-12 and
1 - F <= 1e-12; FP32 (fused tensor cores) 1 - F <= 1e-6.

Samples: two states that differ in their last bits have sequential FP64 prefixes that
differ by a random walk of rounding errors, about sqrt(2^30) * ulp(1)/2 ~ 2e-12 at the
end, while the intervals of a 2^30 state are ~1e-9 wide; so a draw within ~1e-11 of an
end of its interval may pick the neighbour (a few of 4,096 draws).  A draw farther from
the ends must give the reference's sample.  The per-gate engine's state is the
reference's bit for bit, so there every sample must be equal.  The sampling itself is
checked exact on the GPU's own state by test_headline_sampling_exact_at_cdf_edges."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
HALF = 15


def native():
    from svsim_b200 import _native
    return _native


class _DeviceArray:
    """Exposes a device pointer to torch through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_state(h):
    """The handle's state as a complex128 torch tensor on the GPU (a view for FP64, a
    widened copy for FP32)."""
    import torch
    ptr, prec = h.device_ptr()
    nat = native()
    ty = "<f8" if prec == nat.SVB_FP64 else "<f4"
    t = torch.as_tensor(_DeviceArray(ptr, (1 << h.n, 2), ty), device="cuda:0")
    if prec != nat.SVB_FP64:
        t = t.double()
    return torch.view_as_complex(t)


def sketch_signs(rows, seed):
    rng = np.random.default_rng(seed)
    r = rng.integers(0, 2, size=(rows, 1 << HALF)).astype(np.float64) * 2.0 - 1.0
    c = rng.integers(0, 2, size=(rows, 1 << HALF)).astype(np.float64) * 2.0 - 1.0
    return r, c


def gpu_sketch(a, rows, seed):
    import torch
    r, c = sketch_signs(rows, seed)
    rt = torch.from_numpy(r).to(a.device).to(torch.complex128)
    ct = torch.from_numpy(c).to(a.device).to(torch.complex128)
    b = a.reshape(1 << HALF, 1 << HALF) @ ct.T            # [hi, k]
    return (rt * b.T).sum(dim=1).cpu().numpy()


def gpu_checksum(a, chunk=1 << 26):
    import torch
    tot = 0j
    for s in range(0, a.numel(), chunk):
        i = torch.arange(s, min(s + chunk, a.numel()), dtype=torch.float64, device=a.device)
        w = torch.complex(torch.cos(0.7 * i), torch.sin(1.3 * i))
        tot += complex((a[s:s + chunk] * w).sum().item())
    return tot


def compare_with_golden(h, d):
    """(max |d amp| at the fixture's indices, sketch estimate of ||a - a_ref||^2, checksum
    difference, norm difference)."""
    import torch
    a = device_state(h)
    idx = torch.from_numpy(d["idx"].astype(np.int64)).to(a.device)
    at = a[idx].cpu().numpy()
    ref = d["re_at"] + 1j * d["im_at"]
    max_abs = float(np.max(np.abs(at - ref)))
    sk = gpu_sketch(a, int(d["sketch_rows"][0]), int(d["sketch_seed"][0]))
    err2 = float(np.mean(np.abs(sk - d["sketch"]) ** 2))
    cs = abs(gpu_checksum(a) - complex(d["checksum"][0]))
    del a
    torch.cuda.synchronize()
    _, total = h.measure(np.zeros(0))        # the reference's sequential prefix total
    return max_abs, err2, cs, abs(total - float(d["norm"][0]))


def sample_mismatches(h, d, near=1e-10):
    """Shots whose sample differs from the reference's, and how many of those lie within
    `near` of an end of the reference's interval (a rounding-level state difference)."""
    got, _ = h.measure(d["uniforms"])
    bad = np.nonzero(got != d["samples"])[0]
    u = d["uniforms"][bad]
    margin = np.minimum(u - d["sample_lo"][bad], d["sample_hi"][bad] - u)
    return bad.size, int(np.sum(margin < near))


@pytest.fixture(scope="module")
def golden():
    return load_golden("matching_n30.npz")


def run_headline(d, engine, precision=0, fusion_width=0):
    nat = native()
    h = nat.Handle(int(d["n"][0]), 0, precision)
    h.set_engine(engine, 0, fusion_width)
    h.set_circuit(d["gates"])
    h.run()
    h.sync()
    return h


def test_fixture_is_the_bench_circuit(golden):
    from svsim_b200 import circuits
    g = circuits.random_matching_circuit(30, 40, seed=2024)
    assert np.array_equal(golden["gates"], g)


@pytest.mark.parametrize("engine", ["pairs", "staged", "per_gate"])
def test_headline_fp64_matches_reference(golden, engine):
    nat = native()
    eng = {"pairs": nat.ENGINE_PAIRS, "staged": nat.ENGINE_STAGED, "per_gate": nat.ENGINE_PER_GATE}[engine]
    h = run_headline(golden, eng)
    try:
        max_abs, err2, cs, dnorm = compare_with_golden(h, golden)
        print(f"{engine}: max|d amp| {max_abs:.3e}, ||e||^2 (sketch) {err2:.3e}, "
              f"checksum {cs:.3e}, norm {dnorm:.3e}")
        assert max_abs <= FP64_TOL
        assert err2 <= FP64_TOL          # 1 - F <= ||e||^2
        assert cs <= 1e-10
        assert dnorm <= FP64_TOL
        bad, near = sample_mismatches(h, golden)
        print(f"{engine}: {bad} of 4096 samples differ, {near} of them within 1e-10 of a CDF end")
        assert bad == near, (bad, near)
        assert bad <= 40
        if engine == "per_gate":         # the reference's state bit for bit
            assert max_abs == 0.0 and dnorm == 0.0 and bad == 0
    finally:
        h.close()


@pytest.mark.parametrize("k", [4, 5, 6])
def test_headline_fused_fp32_matches_reference(golden, k):
    nat = native()
    h = run_headline(golden, nat.ENGINE_FUSED, precision=nat.SVB_FP32, fusion_width=k)
    try:
        max_abs, err2, cs, dnorm = compare_with_golden(h, golden)
        print(f"fused k={k}: max|d amp| {max_abs:.3e}, ||e||^2 (sketch) {err2:.3e}, "
              f"checksum {cs:.3e}, norm {dnorm:.3e}")
        assert err2 <= 1e-6
        assert max_abs <= 1e-6
    finally:
        h.close()


def test_headline_sampling_exact_at_cdf_edges():
    """Uniforms on the GPU state's own S_j (the reference's sequential prefix of that
    state, from numpy's sequential cumsum) and on their neighbours: the samples equal the
    reference rule's at 2^30 amplitudes, where the prefix crosses many binades and
    4,096 superblocks.  Needs ~32 GiB of host memory for the state and its prefix."""
    import psutil
    if psutil.virtual_memory().available < 48 * 2**30:
        pytest.skip("needs 48 GiB of free host memory")
    nat = native()
    from svsim_b200 import circuits
    h = nat.Handle(30, 0, nat.SVB_FP64)
    h.set_circuit(circuits.random_matching_circuit(30, 40, seed=2024))
    h.run()
    h.sync()
    try:
        re, im = h.get_state()
        p = re * re
        p += im * im
        del re, im
        scan = np.empty(p.size + 1)
        scan[0] = 0.0
        np.cumsum(p, out=scan[1:])
        del p
        rng = np.random.default_rng(30)
        js = rng.choice(1 << 30, size=400, replace=False)
        sj = scan[js]
        u = np.concatenate([sj, np.nextafter(sj, -np.inf), np.nextafter(sj, np.inf),
                            [scan[-1], np.nextafter(scan[-1], -np.inf), 1.0], rng.random(1024)])
        k = np.searchsorted(scan, u, side="right") - 1
        want = np.where((k >= 0) & (k < (1 << 30)), k, 0).astype(np.uint64)
        got, total = h.measure(u)
        assert total == scan[-1]
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, [(float(u[i]), int(got[i]), int(want[i])) for i in bad[:8]]
    finally:
        h.close()
