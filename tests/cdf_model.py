"""A numpy model of the GPU's exact measurement CDF (csrc/measure.cu), for CPU tests.

The reference samples against the sequential FP64 prefix S_0 = 0,
S_{i+1} = fl(S_i + p_i), p_i = fl(fl(re_i^2) + fl(im_i^2)) (svsim_nvgpu_sin.cuh:362-365;
the CPU twins svsim_cpu_sin.hpp:324-346 are identical).  The GPU reproduces that
prefix bit for bit without a sequential pass over 2^n elements: while S stays in one
binade [2^e, 2^(e+1)), every S is an integer multiple of the grid unit u = 2^(e-52),
and fl(S + p) = S + round(p / u) * u unless p / u has a fractional part of exactly
one half (a tie, whose rounding depends on S's last bit) or the sum leaves the binade.
So runs of elements advance S by exact integer sums (parallel), and only ties and
binade crossings are added one by one.  This module restates that arithmetic with
numpy integers (the same bit manipulations as the kernels) so the scheme can be
checked against ``np.cumsum`` (which is sequential, like the reference) on CPU.
"""
from __future__ import annotations

import numpy as np

FRAC = (1 << 52) - 1
M_MAX = (1 << 53) - 1
BLOCK = 4096
CHUNK = 32
SUPER = 64


def probs(re: np.ndarray, im: np.ndarray) -> np.ndarray:
    p = re * re
    p += im * im
    return p


def grid_units(p: np.ndarray, e: int):
    """(d, ok): round(p / 2^(e-52)) per element, ok=False on a tie or a result >= 2^52
    (restates grid_units in csrc/measure.cu)."""
    bits = p.view(np.uint64)
    ebits = ((bits >> np.uint64(52)) & np.uint64(0x7FF)).astype(np.int64)
    mp = bits & np.uint64(FRAC)
    normal = ebits != 0
    mp = np.where(normal, mp | np.uint64(1 << 52), mp)
    ep = np.where(normal, ebits - 1023, -1022)
    sh = e - ep
    d = np.zeros(p.shape, dtype=np.uint64)
    ok = np.ones(p.shape, dtype=bool)
    bad = ebits == 0x7FF
    neg = sh < 0
    ok[neg] = mp[neg] == 0
    zero_sh = sh == 0
    d[zero_sh] = mp[zero_sh]
    ok[zero_sh] &= mp[zero_sh] < np.uint64(1 << 52)
    gen = (sh > 0) & (sh < 64)
    s = sh[gen].astype(np.uint64)
    m = mp[gen]
    ip = m >> s
    fr = m & ((np.uint64(1) << s) - np.uint64(1))
    half = np.uint64(1) << (s - np.uint64(1))
    d[gen] = ip + (fr > half).astype(np.uint64)
    ok[gen] = fr != half
    ok[bad] = False
    return d, ok


def split(t: float):
    """(e, m) with t = m * 2^(e-52), m in [2^52, 2^53), or None when t is not a normal
    positive double."""
    b = int(np.float64(t).view(np.uint64))
    eb = (b >> 52) & 0x7FF
    if b >> 63 or eb == 0 or eb == 0x7FF:
        return None
    return eb - 1023, (b & FRAC) | (1 << 52)


def join(e: int, m: int) -> float:
    return float(np.uint64(((e + 1023) << 52) | (m - (1 << 52))).view(np.float64))


def advance(t: float, e: int, d: int):
    """t + d grid units of binade e, if t lies in that binade and stays there."""
    sm = split(t)
    if sm is None or sm[0] != e or d > M_MAX - sm[1]:
        return None
    return join(e, sm[1] + d)


def chunk_scan(s_in: float, p: np.ndarray) -> np.ndarray:
    """Inclusive sequential prefix of one chunk from s_in, exact (chunk_scan_exact)."""
    sm = split(s_in)
    if sm is not None:
        e, m = sm
        d, ok = grid_units(p, e)
        if ok.all():
            incl = np.cumsum(d.astype(object))
            if incl[-1] <= M_MAX - m:
                return np.array([join(e, m + int(x)) for x in incl])
    out = np.empty(p.size)
    s = s_in
    for k in range(p.size):
        s = float(np.float64(s) + np.float64(p[k]))
        out[k] = s
    return out


def walk(s: float, p: np.ndarray) -> float:
    for c in range(0, p.size, CHUNK):
        s = float(chunk_scan(s, p[c:c + CHUNK])[-1])
    return s


def block_starts(p: np.ndarray):
    """T_b = S at every block start (and the total), by the kernels' passes:
    approximate block sums and prefix, per-block grid deltas for the binade the
    approximate prefix suggests, superblocks of 64 blocks, one chain over superblocks
    (descending into blocks and chunks where a delta does not apply), then a fill."""
    nb = max(1, -(-p.size // BLOCK))
    pp = np.zeros(nb * BLOCK)
    pp[:p.size] = p
    blocks = pp.reshape(nb, BLOCK)
    approx = np.concatenate([[0.0], np.cumsum(blocks.sum(axis=1))])
    info = []                                    # (kind, e, d): kind 'z', 'v', 'x'
    for b in range(nb):
        if not blocks[b].any():
            info.append(("z", 0, 0))
            continue
        sa, sb = split(approx[b]), split(approx[b + 1])
        if sa is None or sb is None or sa[0] != sb[0]:
            info.append(("x", 0, 0))
            continue
        d, ok = grid_units(blocks[b], sa[0])
        tot = int(d.astype(object).sum())
        info.append(("v", sa[0], tot) if ok.all() and tot < (1 << 52) else ("x", 0, 0))
    nsb = -(-nb // SUPER)
    sinfo = []
    for s in range(nsb):
        ks = info[s * SUPER:(s + 1) * SUPER]
        nz = [k for k in ks if k[0] != "z"]
        if not nz:
            sinfo.append(("z", 0, 0))
        elif all(k[0] == "v" for k in nz) and len({k[1] for k in nz}) == 1 \
                and sum(k[2] for k in nz) < (1 << 52):
            sinfo.append(("v", nz[0][1], sum(k[2] for k in nz)))
        else:
            sinfo.append(("x", 0, 0))
    T = np.zeros(nb + 1)
    t = 0.0
    for s in range(nsb):
        kind, e, d = sinfo[s]
        if kind == "z":
            T[s * SUPER:min((s + 1) * SUPER, nb)] = t
            continue
        if kind == "v":
            nt = advance(t, e, d)
            if nt is not None:
                for b in range(s * SUPER, min((s + 1) * SUPER, nb)):      # the fill
                    T[b] = t
                    if info[b][0] == "v":
                        t = advance(t, info[b][1], info[b][2])
                assert t == nt
                continue
        for b in range(s * SUPER, min((s + 1) * SUPER, nb)):
            T[b] = t
            k = info[b]
            if k[0] == "z":
                continue
            nt = advance(t, k[1], k[2]) if k[0] == "v" else None
            t = nt if nt is not None else walk(t, blocks[b])
    T[nb] = t
    return T, blocks


def sample(re: np.ndarray, im: np.ndarray, uniforms) -> np.ndarray:
    """The reference's samples for `uniforms`, by the GPU's scheme."""
    p = probs(re, im)
    T, blocks = block_starts(p)
    dim = p.size
    out = np.zeros(len(uniforms), dtype=np.uint64)
    for k, r in enumerate(uniforms):
        if not (r >= 0.0 and r < T[-1]):
            continue
        b = int(np.searchsorted(T[:-1], r, side="right") - 1)
        s = T[b]
        found = None
        for c in range(0, BLOCK, CHUNK):
            incl = chunk_scan(s, blocks[b, c:c + CHUNK])
            hit = np.nonzero(incl > r)[0]
            if hit.size:
                found = b * BLOCK + c + int(hit[0])
                break
            s = float(incl[-1])
        assert found is not None and found < dim
        out[k] = found
    return out


def reference_samples(re: np.ndarray, im: np.ndarray, uniforms) -> np.ndarray:
    """The rule of svsim_cpu_sin.hpp:324-346 on np.cumsum (sequential in index order)."""
    p = probs(re, im)
    scan = np.concatenate([[0.0], np.cumsum(p)])
    r = np.asarray(uniforms, dtype=np.float64)
    k = np.searchsorted(scan, r, side="right") - 1
    return np.where((k >= 0) & (k < p.size), k, 0).astype(np.uint64)
