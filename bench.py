#!/usr/bin/env python
"""Benchmark of the B200 state-vector engine.

Workload (one "step"): the n=30, depth-40 random circuit — per layer U3 with U[0,2pi)
angles on all 30 qubits, then 15 CX on a seeded random perfect matching (1,800 gates) —
applied in FP64 to a 16 GiB state resident in HBM, through the pair engine (two-qubit
blocks on the FP64 tensor cores).  The state (16 GiB) is far larger than the 126 MB L2, so
no L2 flush is needed between steps.

Printed (rank 0, one JSON line): gates/s over all ranks, the roofline of the dominant
kernel (`k_pairs`: HBM bytes per launch and its FP64 tensor-pipe rate beside them), the
reference CPU path timed on this box's
host cores, an end-to-end figure through the C ABI with host buffers, the SM clocks seen
during the timed region, and secondary forms (per-gate FP64 sweeps, adjoint gradients).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs the same workload on its own GPU: a single circuit
does not shard without an exchange step, so the multi-GPU figure is N replicas.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sv-sim_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

N_QUBITS = 30
DEPTH = 40
SEED = 2024
FUSION_WIDTH = 5        # qubits per fused block of the tensor-core FP32 form
METRIC = "n=30 gates/s & HBM GB/s: FP64 per-gate vs fused TC (1-F≤1e-6); adjoint grads/s"
UNIT = "gates/s"
WORKLOAD = "random circuit n=30 depth 40 (U3 all qubits + 15 CX random matching per layer), FP64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-extras", action="store_true", help="skip the secondary forms")
    ap.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--qubits", type=int, default=N_QUBITS,
                    help="state size (smaller cases are for profiling only)")
    ap.add_argument("--tile-bits", type=int, default=12)
    ap.add_argument("--engine", choices=["staged", "pairs"], default="pairs",
                    help="FP64 engine of the headline step")
    ap.add_argument("--form", choices=["headline", "pergate", "fused", "qaoa", "capacity", "adjoint", "density",
                                       "config1", "tuning", "batch", "refgpu"],
                    default="headline",
                    help="headline: the FP64 n=30 step (the measured line); the others run one "
                         "secondary form alone (for profiling and capacity runs)")
    ap.add_argument("--instances", type=int, default=512, help="QAOA batch size (--form qaoa)")
    ap.add_argument("--fusion-width", type=int, default=FUSION_WIDTH, choices=[3, 4, 5, 6],
                    help="qubits per fused block of the tensor-core FP32 form")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64",
                    help="state precision of --form qaoa")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_sample_gates(circuit):
    """The bounded CPU sample: every third gate of the first layer (15 of its 45 gates:
    10 U3 spread over low and high qubits and 5 CX), applied to the 30-qubit state."""
    return circuit[:45][::3].copy()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.reader.join(timeout=2)

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_rate(circuit, threads):
    """gates/s of the reference's OpenMP CPU backend on the bounded sample."""
    from oracle.oracle import RefBackend
    sample = cpu_sample_gates(circuit)
    kind, backend = "reference", None
    for k in ("omp64",):
        if RefBackend.available(k):
            backend = RefBackend(k)
    if backend is None:
        return None
    h = backend.open(N_QUBITS, threads)
    try:
        ms = backend.run_on(h, sample)
    finally:
        backend.close(h)
    return {"value": len(sample) / (ms / 1e3), "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{len(sample)} gates of layer 1 (every 3rd) at n=30, reference "
                      f"svsim_cpu_omp.hpp (64-bit IdxType build), sim() wall time {ms:.0f} ms"}


class _DeviceArray:
    """A device pointer seen by torch through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def golden_parity(h):
    """The handle's state (the n=30 circuit run once from |0..0>) against the reference's
    own cpu_omp state of the same circuit, through tests/golden/matching_n30.npz: the
    largest amplitude error at the fixture's 4,097 indices, the sketch estimate of
    ||a - a_ref||^2 (>= 1 - F), and how many of the fixture's 4,096 reference-rule samples
    svb_measure reproduces for the same draws."""
    import torch
    from svsim_b200 import _native as nat
    path = os.path.join(ROOT, "tests", "golden", "matching_n30.npz")
    if not os.path.exists(path):
        return None
    d = np.load(path)
    ptr, prec = h.device_ptr()
    t = torch.as_tensor(_DeviceArray(ptr, (1 << h.n, 2), "<f8" if prec == nat.SVB_FP64 else "<f4"),
                        device=f"cuda:{torch.cuda.current_device()}")
    a = torch.view_as_complex(t if prec == nat.SVB_FP64 else t.double())
    idx = torch.from_numpy(d["idx"].astype(np.int64)).to(a.device)
    max_abs = float(np.max(np.abs(a[idx].cpu().numpy() - (d["re_at"] + 1j * d["im_at"]))))
    rows, seed = int(d["sketch_rows"][0]), int(d["sketch_seed"][0])
    rng = np.random.default_rng(seed)
    r = rng.integers(0, 2, size=(rows, 1 << 15)).astype(np.float64) * 2.0 - 1.0
    c = rng.integers(0, 2, size=(rows, 1 << 15)).astype(np.float64) * 2.0 - 1.0
    rt = torch.from_numpy(r).to(a.device).to(torch.complex128)
    ct = torch.from_numpy(c).to(a.device).to(torch.complex128)
    sk = (rt * (a.reshape(1 << 15, 1 << 15) @ ct.T).T).sum(dim=1).cpu().numpy()
    del a, t
    err2 = float(np.mean(np.abs(sk - d["sketch"]) ** 2))
    samples, total = h.measure(d["uniforms"])
    return {"reference": "svsim_cpu_omp.hpp (64-bit IdxType build) state of the same circuit, "
                         "tests/golden/matching_n30.npz",
            "max_abs_err_vs_reference": max_abs, "amplitudes_compared": int(d["idx"].size),
            "infidelity_bound_vs_reference": err2,
            "infidelity_bound_how": f"mean |c_k(a) - c_k(a_ref)|^2 over {rows} random-sign projections "
                                    "(estimates ||a - a_ref||^2 >= 1 - F)",
            "norm_diff_vs_reference": abs(total - float(d["norm"][0])),
            "samples_equal_to_reference": int(np.sum(samples == d["samples"])),
            "samples_compared": int(d["samples"].size)}


def dropin_e2e(circuit, device, steps, world):
    """The same metric through the reference's own Python front end: the libsvsim module
    compiled from svsim/src/py_wrapper.cpp against the drop-in headers.  Each step is
    upload() + run() + measure(1024), the calls a reference user makes; the gates are
    appended once (the user's circuit construction).  sim() no longer copies the 16 GiB
    state back, so nothing but the gate records, the plan and the samples crosses PCIe."""
    import torch
    lib = os.path.join(ROOT, "sv-sim_b200", "svsim_b200", "lib")
    if not os.path.isdir(lib) or not any(f.startswith("libsvsim.") for f in os.listdir(lib)):
        return None
    sys.path.insert(0, lib)
    import libsvsim
    from svsim_b200 import gates as G
    sim = libsvsim.Simulation(N_QUBITS, device)
    for g in circuit:
        op, qb = int(g["op"]), g["qb"]
        if op == G.OP["U3"]:
            sim.append(sim.U3(float(g["theta"]), float(g["phi"]), float(g["lam"]), int(qb[0])))
        else:
            sim.append(sim.CX(int(qb[0]), int(qb[1])))
    sim.upload()
    sim.run()
    sim.measure(1024)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.upload()
        sim.run()
        res = sim.measure(1024)
    torch.cuda.synchronize(device)
    dt = (time.perf_counter() - t0) / steps
    del sim
    if world > 1:
        t = torch.tensor([dt], dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        dt = float(t.item())
    return {"value": world * len(circuit) / dt, "unit": UNIT, "s_per_step": dt,
            "h2d_bytes_per_step": int(circuit.nbytes), "d2h_bytes_per_step": int(8 * len(res) + 8),
            "path": "libsvsim (svsim/src/py_wrapper.cpp built against the drop-in headers): "
                    "upload() + run() + measure(1024)"}


def run_reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from svsim_b200 import circuits
    from oracle.oracle import RefBackend
    circuit = circuits.random_matching_circuit(N_QUBITS, DEPTH, seed=SEED)
    threads = os.cpu_count() or 1
    if not RefBackend.available("omp64"):
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU backend not built (oracle/_ref missing)"}))
        return
    sample = cpu_sample_gates(circuit)
    backend = RefBackend("omp64")
    h = backend.open(N_QUBITS, threads)
    for _ in range(args.warmup):
        backend.run_on(h, sample)
    times = [backend.run_on(h, sample) for _ in range(args.steps)]
    backend.close(h)
    total_s = sum(times) / 1e3
    value = len(sample) * args.steps / total_s
    sample_desc = (f"{len(sample)} gates of layer 1 (every 3rd) at n=30 per step, reference "
                   f"svsim_cpu_omp.hpp (64-bit IdxType build), {threads} threads")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_qubits": N_QUBITS, "depth": DEPTH, "seed": SEED,
                   "sample": sample_desc},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample_desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ours(args):
    import torch
    from svsim_b200 import circuits, _native as nat

    world, rank, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    device = local
    torch.cuda.set_device(device)
    nq = args.qubits
    circuit = circuits.random_matching_circuit(nq, DEPTH, seed=SEED)
    n_gates = len(circuit)

    h = nat.Handle(nq, device, nat.SVB_FP64)
    if args.engine == "pairs":
        h.set_engine(nat.ENGINE_PAIRS, 0, 0)
    else:
        h.set_engine(nat.ENGINE_STAGED, args.tile_bits, 0)
    h.set_circuit(circuit)
    info = h.plan_info()
    stream = torch.cuda.current_stream(device)
    sptr = stream.cuda_stream

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(max(args.warmup, 3)):
        h.run(sptr)
    torch.cuda.synchronize(device)
    barrier()
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            h.run(sptr)
        ev1.record(stream)
        torch.cuda.synchronize(device)
    barrier()
    torch.cuda.synchronize(device)
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = world * n_gates * args.steps / (ms / 1e3)

    # roofline of the dominant kernel: every staged pass reads and writes the state once
    state_bytes = info.state_bytes
    passes = int(info.n_passes)
    per_launch_bytes = 2.0 * state_bytes
    launch_s = (ms / 1e3) / (args.steps * passes)
    achieved = per_launch_bytes / launch_s / 1e9
    peak, peak_kind = peaks()
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "pairs_fp64_traffic.txt" if args.engine == "pairs"
                         else "staged_fp64_traffic.txt")
    if os.path.exists(tfile):
        for ln in open(tfile):
            if ln.startswith("bytes_per_launch_n30"):
                traffic = float(ln.split("=")[1])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": ("k_pairs (FP64 mma.sync two-qubit blocks)" if args.engine == "pairs"
                           else "k_staged<double,12>") + f" (one read+write of the {16 << nq >> 30} GiB state per launch)",
                "peak_source": f"{peak_kind} hbm_gbs",
                "per_launch_bytes": per_launch_bytes, "launches_per_step": passes,
                "gate_model_gbs": info.model_bytes / (ms_per_step / 1e3) / 1e9}
    if args.engine == "pairs" and int(info.n_blocks) > 0:
        # the pair kernel is bound by the FP64 tensor cores, not by HBM: each two-qubit
        # block is 16 multiply-adds per amplitude; the rate they allow is measured live
        flops = int(info.n_blocks) * float(1 << nq) * 16 * 2
        tf = flops / (ms_per_step / 1e3) / 1e12
        tf_peak = nat.fp64_mma_peak(device)
        roofline["fp64_tensor"] = {"achieved": tf, "peak": tf_peak, "unit": "TFLOP/s", "frac": tf / tf_peak,
                                   "blocks_per_step": int(info.n_blocks),
                                   "peak_source": "svb_fp64_mma_peak: register-only mma.sync m8n8k4 f64 loop, "
                                                  "measured in this run"}

    # end to end through the C ABI with host buffers: circuit upload + plan, run,
    # 1024-shot measurement back to host
    shots = 1024
    uni = np.random.default_rng(0).random(shots)
    pinned_gates = torch.from_numpy(circuit.view(np.uint8).copy()).pin_memory()
    e2e_steps = max(2, min(args.steps, 3))
    torch.cuda.synchronize(device)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        h.set_circuit(pinned_gates.numpy().view(circuit.dtype))
        h.run(sptr)
        samples, _tot = h.measure(uni)
    torch.cuda.synchronize(device)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:                      # the slowest rank sets the whole job's rate
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * n_gates / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(circuit.nbytes + info.plan_bytes + uni.nbytes),
           "d2h_bytes_per_step": int(samples.nbytes + 8),
           "path": "svb_set_circuit + svb_run + svb_measure(1024 shots), host buffers"}

    e2e_dropin = dropin_e2e(circuit, device, e2e_steps, world) if nq == N_QUBITS else None
    if e2e_dropin:
        e2e["dropin"] = e2e_dropin

    parity = None
    if nq == N_QUBITS and rank == 0:
        h.reset()
        h.set_circuit(circuit)
        h.run(sptr)
        torch.cuda.synchronize(device)
        parity = golden_parity(h)

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_qubits": nq, "depth": DEPTH, "gates": n_gates,
                   "seed": SEED, "engine": args.engine, "tile_bits": int(info.tile_bits),
                   "passes": passes, "parallelism": f"replicas x{world}",
                   "l2": f"{16 << nq >> 30} GiB state > 126 MB L2: every step streams from HBM, no flush"},
        "roofline": roofline,
        "parity": parity,
        "e2e": e2e,
        "clocks": clocks.summary(),
        "gpu_launches": int(args.steps * passes),
    }
    del h
    torch.cuda.empty_cache()

    if nq != N_QUBITS:
        out["config"]["workload"] = f"profiling case: n={nq} (not the headline workload)"
    if rank == 0 and world == 1 and not args.no_baseline and nq == N_QUBITS:
        threads = os.cpu_count() or 1
        try:
            out["cpu_baseline"] = cpu_reference_rate(circuit, threads)
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"value": None, "error": str(e)}
    if rank == 0 and not args.no_extras and world == 1 and nq == N_QUBITS:
        out["forms"] = secondary_forms(device, circuit)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def qaoa_form(device, count=512, precision="fp64", reps=5):
    """Batched QAOA: energy and gradient of every instance per evaluation; kernel timed
    alone on the device (parameters resident) and end to end through svb_qaoa_run (host
    parameters in, host energies and gradients out)."""
    import torch
    from svsim_b200 import circuits, _native as nat
    insts = circuits.qaoa_instances(count)
    g = np.stack([i.gammas for i in insts])
    b = np.stack([i.betas for i in insts])
    prec = nat.SVB_FP64 if precision == "fp64" else nat.SVB_FP32
    B = nat.QaoaBatch(insts, device, prec)
    st = B.info()
    B.run(g, b)
    s = torch.cuda.Stream(device)
    for _ in range(3):
        B.launch(s.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    e0.record(s)
    for _ in range(reps):
        B.launch(s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize(device)
    sec = e0.elapsed_time(e1) / 1e3 / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        B.run(g, b)
    e2e = (time.perf_counter() - t0) / reps
    B.close()
    torch.cuda.empty_cache()
    peak, kind = peaks()
    return {"instances_per_s": count / sec, "ms_per_batch": sec * 1e3,
            "e2e_instances_per_s": count / e2e, "e2e_ms_per_batch": e2e * 1e3,
            "hbm_gbs": st.moved_bytes / sec / 1e9, "frac_of_peak": st.moved_bytes / sec / 1e9 / peak,
            "moved_bytes_per_batch": st.moved_bytes, "total_amplitudes": int(st.total_amplitudes),
            "tiles_per_pass": int(st.tiles_per_pass), "graphed": bool(st.graphed),
            "precision": precision, "p": int(st.p), "grid": int(st.grid),
            "e2e_h2d_bytes": int(g.nbytes + b.nbytes), "e2e_d2h_bytes": int(count * (1 + 2 * st.p) * 8 + 4),
            "kernel": "k_qaoa (one cooperative launch: 4p tile passes, grid barriers between)",
            "workload": f"{count} MaxCut instances, n ~ U{{10..22}}, G(n,0.3), p=4"}


def capacity_form(device, shots=4096):
    """The largest states of one B200: n=33 FP64 (pair engine, 128 GiB) and n=34 FP32 (fused,
    128 GiB), depth-20 random-matching circuits, 4096-shot sampling with the FP64 CDF."""
    import torch
    from svsim_b200 import circuits, _native as nat
    out = {}
    uni = np.random.default_rng(1).random(shots)
    for n, prec, eng, k, name in ((33, nat.SVB_FP64, nat.ENGINE_PAIRS, 0, "n33_fp64_pairs"),
                                  (34, nat.SVB_FP32, nat.ENGINE_FUSED, 5, "n34_fp32_fused")):
        circ = circuits.random_matching_circuit(n, 20, seed=SEED)
        h = nat.Handle(n, device, prec)
        h.set_engine(eng, 0, k)
        h.set_circuit(circ)
        info = h.plan_info()
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        h.run()
        e1.record()
        torch.cuda.synchronize(device)
        h.sync()
        sec = e0.elapsed_time(e1) / 1e3
        t0 = time.perf_counter()
        samples, total = h.measure(uni)
        t_meas = time.perf_counter() - t0
        out[name] = {"gates_per_s": len(circ) / sec, "s_per_circuit": sec, "passes": int(info.n_passes),
                     "state_gib": info.state_bytes / 2**30, "hbm_gbs": info.moved_bytes / sec / 1e9,
                     "shots": shots, "measure_s": t_meas, "prob_total": total,
                     "distinct_outcomes": int(len(np.unique(samples)))}
        del h
        torch.cuda.empty_cache()
    return out


def qaoa_sharded_form(args, world, rank, local):
    """Batched QAOA split over the ranks (one GPU each, size-balanced, results gathered by
    one all-reduce).  Each step is one full evaluation through ShardedQaoa.run with host
    parameters in and host results out; the time is the max over ranks."""
    import datetime
    import torch
    import torch.distributed as dist
    from svsim_b200 import circuits, _native as nat
    from svsim_b200.sharding import ShardedQaoa
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    insts = circuits.qaoa_instances(args.instances)
    g = np.stack([i.gammas for i in insts])
    b = np.stack([i.betas for i in insts])
    prec = nat.SVB_FP64 if args.precision == "fp64" else nat.SVB_FP32
    sq = ShardedQaoa(insts, device=local, precision=prec)
    for _ in range(max(args.warmup, 3)):
        sq.run(g, b)
    dist.barrier()
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sq.run(g, b)
    torch.cuda.synchronize(local)
    dt = time.perf_counter() - t0
    t = torch.tensor([dt], device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dt = float(t.item())
    mine_amps = sum(1 << insts[i].n for i in sq.mine)
    sq.close()
    dist.barrier()
    dist.destroy_process_group()
    return {"form": "qaoa", "instances_per_s": args.instances * args.steps / dt,
            "ms_per_batch": dt / args.steps * 1e3, "n_gpus": world, "precision": args.precision,
            "scaling": "strong", "rank0_instances": len(sq.mine), "rank0_amplitudes": mine_amps,
            "path": "ShardedQaoa.run: host parameters in, per-rank svb_qaoa_run, all-reduce gather"}


def run_form(args):
    """One secondary form alone, as one JSON line (rank 0 prints)."""
    import torch
    world, rank, local = dist_env()
    if args.form == "qaoa" and world > 1:
        res = qaoa_sharded_form(args, world, rank, local)
        if rank == 0:
            print(json.dumps(res))
        return
    if rank != 0:
        return
    torch.cuda.set_device(local)
    if args.form == "adjoint":
        res = adjoint_form(local, reps=max(1, args.steps), warmup=args.warmup, shift=not args.no_baseline)
    elif args.form == "density":
        res = density_form(local)
    elif args.form == "config1":
        res = config1_form(local)
    elif args.form == "tuning":
        res = tuning_form(local)
    elif args.form == "batch":
        res = batch_form(local)
    elif args.form == "refgpu":
        res = reference_gpu_form(local)
    elif args.form == "pergate":
        from svsim_b200 import circuits
        res = per_gate_form(local, circuits.random_matching_circuit(args.qubits, DEPTH, seed=SEED), n=args.qubits)
    elif args.form == "fused":
        circuit = None
        from svsim_b200 import circuits
        circuit = circuits.random_matching_circuit(args.qubits, DEPTH, seed=SEED)
        res = fused_form(local, circuit, k=args.fusion_width, n=args.qubits, reps=max(1, args.steps))
    elif args.form == "qaoa":
        res = qaoa_form(local, args.instances, args.precision, reps=max(1, args.steps))
    else:
        res = capacity_form(local)
    print(json.dumps({"form": args.form, **res}))


def per_gate_form(device, circuit, n=N_QUBITS):
    """The per-gate FP64 engine (one HBM sweep per elementary op, as the reference) on the
    whole circuit, timed with CUDA events, with the roofline of its two kernels: a dense
    gate (k_eop_pairs) reads and writes the state once, a CX (k_cx) its control = 1 half."""
    import torch
    from svsim_b200 import _native as nat
    h = nat.Handle(n, device, nat.SVB_FP64)
    h.set_engine(nat.ENGINE_PER_GATE, 0, 0)
    h.set_circuit(circuit)
    info = h.plan_info()
    h.run()                                        # warm-up (first launches, clocks)
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    h.run()
    e1.record()
    torch.cuda.synchronize(device)
    h.sync()
    s = e0.elapsed_time(e1) / 1e3
    peak, kind = peaks()
    del h
    torch.cuda.empty_cache()
    achieved = info.moved_bytes / s / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "per_gate_fp64_traffic.txt")
    if os.path.exists(tfile):
        vals = {}
        for ln in open(tfile):
            if "=" in ln and not ln.startswith("#"):
                k, v = ln.split("=", 1)
                vals[k.strip()] = float(v)
        if n == N_QUBITS and "dense_bytes_per_launch_n30" in vals:
            traffic = {"k_eop_pairs_dense": vals["dense_bytes_per_launch_n30"],
                       "k_cx": vals.get("cx_bytes_per_launch_n30")}
    sb = info.state_bytes
    return {"gates_per_s": len(circuit) / s, "s_per_circuit": s, "gates": len(circuit),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{kind} hbm_gbs",
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": {"k_eop_pairs_dense": 2 * sb, "k_cx": sb},
                         "bytes_per_circuit": info.moved_bytes},
            "sample": f"the whole circuit ({len(circuit)} gates), one launch per elementary gate",
            "kernels": "k_eop_pairs / k_cx (4 pairs per thread in flight, 128-bit loads)"}


def config1_form(device, reps=200):
    """The reference's CPU-runnable case: n=16 brickwork, 20 layers (320 U3 + 150 CX =
    470 gates).  The 1 MiB state stays in L2, so each engine is reported against the L2
    copy bandwidth measured in this run; beside it the reference's cpu_sin on one core
    and cpu_omp on every host core run the same circuit."""
    import torch
    from svsim_b200 import circuits, _native as nat
    g = circuits.brickwork_circuit(16, 20, seed=1234)
    l2 = nat.l2_copy_peak(device)
    out = {"workload": "brickwork n=16, 20 layers, 470 gates, FP64", "l2_copy_peak_gbs": l2,
           "l2_peak_source": "svb_l2_copy_peak: 2 x 16 MiB copy repeated in one launch, this run"}
    gold = np.load(os.path.join(ROOT, "tests", "golden", "brickwork.npz"))
    for name, eng in (("pairs", nat.ENGINE_PAIRS), ("staged", nat.ENGINE_STAGED), ("per_gate", nat.ENGINE_PER_GATE)):
        h = nat.Handle(16, device, nat.SVB_FP64)
        h.set_engine(eng, 0, 0)
        h.set_circuit(g)
        info = h.plan_info()
        h.run()
        re, im = h.get_state()
        err = float(np.max(np.abs((re + 1j * im)[gold["idx16"]] - (gold["re16_at"] + 1j * gold["im16_at"]))))
        for _ in range(5):
            h.run()
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            h.run()
        e1.record()
        torch.cuda.synchronize(device)
        h.sync()
        sec = e0.elapsed_time(e1) / 1e3 / reps
        out[name] = {"gates_per_s": len(g) / sec, "us_per_circuit": sec * 1e6,
                     "launches": int(info.n_passes), "l2_gbs": info.moved_bytes / sec / 1e9,
                     "l2_frac": info.moved_bytes / sec / 1e9 / l2,
                     "max_abs_err_vs_reference": err}
        h.close()
    try:
        from oracle.oracle import RefBackend
        threads = os.cpu_count() or 1
        for kind, th, key in (("sin", 1, "reference_cpu_sin_1core"), ("omp", threads, "reference_cpu_omp_all_cores")):
            if RefBackend.available(kind):
                ref = RefBackend(kind)
                ms = min(ref.simulate(16, g, threads=th, want_state=False)["sim_ms"] for _ in range(3))
                out[key] = {"gates_per_s": len(g) / (ms / 1e3), "ms_per_circuit": ms, "cores": th}
    except Exception as e:      # the CPU rates are reported, never required
        out["reference_cpu_error"] = str(e)
    return out


def fused_form(device, circuit, k=None, reps=3, n=N_QUBITS):
    """The same circuit on an FP32 state through the fused tensor-core engine, with its
    infidelity bound and largest amplitude error against the reference's FP64 state
    (golden fixture of the reference's cpu_omp)."""
    import torch
    k = FUSION_WIDTH if k is None else k
    from svsim_b200 import _native as nat
    h32 = nat.Handle(n, device, nat.SVB_FP32)
    h32.set_engine(nat.ENGINE_FUSED, 0, k)
    h32.set_circuit(circuit)
    info = h32.plan_info()
    h32.run()
    h32.sync()
    par = golden_parity(h32) if n == N_QUBITS else None
    norm32 = h32.norm2()
    h32.run()
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        h32.run()
    e1.record()
    torch.cuda.synchronize(device)
    h32.sync()
    s = e0.elapsed_time(e1) / 1e3 / reps
    peak, _ = peaks()
    out = {"gates_per_s": len(circuit) / s, "ms_per_circuit": s * 1e3, "fusion_width": k,
           "passes": int(info.n_passes), "blocks": int(info.n_blocks), "hbm_gbs": info.moved_bytes / s / 1e9,
           "hbm_frac_of_peak": info.moved_bytes / s / 1e9 / peak,
           "norm_minus_one": norm32 - 1.0,
           "kernel": f"k_fused<{k}>: split-TF32 tcgen05.mma, M=128, K={2 << k} in steps of 8, "
                     f"N={4 << k} (X_hi [G_hi|G_lo]) + N={2 << k} (X_lo G_hi); A operand and "
                     "accumulators in TMEM, two tiles in flight"}
    if par:
        out["one_minus_fidelity_bound_vs_reference"] = par["infidelity_bound_vs_reference"]
        out["max_abs_amp_err_vs_reference"] = par["max_abs_err_vs_reference"]
        out["samples_equal_to_reference"] = par["samples_equal_to_reference"]
    del h32
    torch.cuda.empty_cache()
    return out


def tuning_form(device):
    """The autotuner on the headline circuit (FP64 and FP32 states of n=30): the candidate
    engines timed on the first 360 gates, the choice next to the static default."""
    import torch
    from svsim_b200 import circuits, _native as nat
    g = circuits.random_matching_circuit(N_QUBITS, DEPTH, seed=SEED)
    names = {0: "auto", 1: "per_gate", 2: "staged", 3: "fused", 4: "pairs"}
    out = {}
    for prec, key in ((nat.SVB_FP64, "fp64"), (nat.SVB_FP32, "fp32")):
        h = nat.Handle(N_QUBITS, device, prec)
        t0 = time.perf_counter()
        r = h.autotune(g)
        out[key] = {"chosen": names.get(r.engine, r.engine), "tile_bits": r.tile_bits,
                    "fusion_width": r.fusion_width, "candidates": r.candidates,
                    "chosen_ms_on_prefix": r.best_ms, "default_ms_on_prefix": r.default_ms,
                    "timed_gates": int(r.timed_gates), "tuning_s": time.perf_counter() - t0}
        h.close()
        torch.cuda.empty_cache()
    return out


def batch_form(device, reps=5):
    """Batched circuits in one graph-replayed persistent launch (svb_cbatch_*): 64
    parameter points of the n=20, 480-parameter ansatz with their energies, and 128
    random circuits with n ~ U{10..22}; the autotuned choice next to the fixed shared-memory
    sweep (12-qubit tiles, 512 threads) and the pair engine (FP64 tensor-core blocks for the
    circuits of 12 or more qubits, the sweep for the rest)."""
    import torch
    from svsim_b200 import circuits, _native as nat
    pc = circuits.hardware_efficient_ansatz()
    terms = circuits.zz_x_hamiltonian(20)
    pts = np.random.default_rng(5).uniform(-np.pi, np.pi, size=(64, len(pc.params)))
    rng = np.random.default_rng(6)
    mixed = []
    for i in range(128):
        n = int(rng.integers(10, 23))
        mixed.append((n, circuits.random_matching_circuit(n, 10, seed=1000 + i)))
    out = {}
    for name, batch, tb in (("ansatz_points_64", [(20, pc.evaluated(p)) for p in pts], None),
                            ("random_mixed_128", mixed, None)):
        res = {}
        for label, tile in (("tuned", 0), ("fixed_tile12", 12), ("pairs", nat.CBATCH_PAIRS)):
            t0 = time.perf_counter()
            b = nat.CircuitBatch(batch, [terms] * len(batch) if name.startswith("ansatz") else None,
                                 device=device, tile_bits=tile)
            setup = time.perf_counter() - t0
            b.run()
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            for _ in range(reps):
                b.run()
            sec = (time.perf_counter() - t0) / reps
            st = b.info()
            gates = sum(len(g) for _, g in batch)
            res[label] = {"circuits_per_s": len(batch) / sec, "ms_per_batch": sec * 1e3,
                          "gates_per_s": gates / sec, "tile_bits": int(st.tile_bits), "threads": int(st.threads),
                          "phases": int(st.n_phases), "graphed": bool(st.graphed), "grid": int(st.grid),
                          "state_gbs": st.moved_bytes / sec / 1e9, "setup_s": setup,
                          "pair_circuits": int(st.pair_circuits)}
            b.close()
            torch.cuda.empty_cache()
        out[name] = res
    out["timing"] = "wall clock of svb_cbatch_run (graph replay, energies back to the host)"
    return out


def reference_gpu_form(device, reps=10):
    """Context only (the timed reference arm is the CPU path): the reference's own
    single-GPU kernel (svsim/src/svsim_nvgpu_sin.cuh, built for sm_100a by oracle/Makefile
    into oracle/_ref/ref_gpu_driver) on this B200, timed by its own event timer around
    the cooperative kernel (sim() prints it), beside this engine on the same circuits:
    the n=16 brickwork (470 gates) and the n=26 random-matching circuit, depth 40."""
    import tempfile
    from svsim_b200 import circuits
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_driver")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_gpu_driver not built (reference tree absent at build time)"}
    out = {}
    for name, n, g in (("brickwork_n16", 16, circuits.brickwork_circuit(16, 20, seed=1234)),
                       ("matching_n26_depth40", 26, circuits.random_matching_circuit(26, DEPTH, seed=SEED))):
        with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
            g.tofile(f)
            path = f.name
        try:
            env = dict(os.environ, CUDA_VISIBLE_DEVICES=str(device))
            r = subprocess.run([exe, path, str(n), str(reps)], capture_output=True, text=True, timeout=300, env=env)
        finally:
            os.unlink(path)
        ms = [float(x.split("sim:")[1].split("ms")[0]) for x in r.stdout.splitlines() if "sim:" in x]
        if r.returncode != 0 or not ms:
            out[name] = {"error": f"rc={r.returncode}", "stderr": r.stderr[-300:]}
            continue
        best = float(np.median(ms[1:] if len(ms) > 1 else ms))
        out[name] = {"gates": len(g), "ms_per_circuit": best, "gates_per_s": len(g) / (best / 1e3),
                     "runs": len(ms)}
    out["what"] = ("reference svsim_nvgpu_sin.cuh compiled for sm_100a (its config.mk flags); "
                   "sim() event time of the cooperative kernel, median of the runs after the first")
    return out


def density_form(device, n=14, depth=10, reps=3):
    """Density matrix of n=14 qubits (a 28-qubit FP64 vector, 4 GiB) through a depth-10
    random-matching circuit with a depolarizing channel (p = 0.01) after every gate on each
    qubit it touches; superoperator blocks on the pair engine."""
    import torch
    from svsim_b200 import circuits, density as D
    g = circuits.random_matching_circuit(n, depth, seed=SEED)
    dm = D.DensityMatrix(n, device)
    dm.set_circuit(g, D.depolarizing(0.01))
    info = dm.plan_info()
    dm.run()
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        dm.handle.run()
    e1.record()
    torch.cuda.synchronize(device)
    sec = e0.elapsed_time(e1) / 1e3 / reps
    dm.reset()                                       # one fresh run for the trace and purity
    dm.run()
    p = dm.probabilities()
    peak, _ = peaks()
    out = {"gates_per_s": len(g) / sec, "ms_per_circuit": sec * 1e3, "passes": int(info.n_passes),
           "engine": int(info.engine), "hbm_gbs": info.moved_bytes / sec / 1e9,
           "frac_of_peak": info.moved_bytes / sec / 1e9 / peak, "trace": float(p.sum()),
           "purity": dm.handle.norm2(),
           "workload": f"rho of n={n} (2n={2 * n} vector qubits), depth {depth}, depolarizing 0.01"}
    dm.close()
    torch.cuda.empty_cache()
    return out


def adjoint_form(device, reps=5, warmup=1, shift=True):
    """Adjoint gradients of the n=20, 480-parameter ansatz (svb_adjoint, wall clock per
    call: host lowering and planning included) against parameter shift on the same GPU
    (2 circuits per parameter, timed on 48 of 480 and scaled; skipped with shift=False)."""
    from svsim_b200 import circuits, _native as nat
    pc = circuits.hardware_efficient_ansatz()
    terms = circuits.zz_x_hamiltonian(20)
    ha = nat.Handle(20, device, nat.SVB_FP64)
    for _ in range(max(1, warmup)):
        ha.adjoint(pc.gates, pc.binding, 480, terms)
    t0 = time.perf_counter()
    for _ in range(reps):
        ha.adjoint(pc.gates, pc.binding, 480, terms)
    t_adj = (time.perf_counter() - t0) / reps
    out = {"grads_per_s": 1.0 / t_adj, "ms_per_gradient": t_adj * 1e3,
           "workload": "n=20, 12 layers RY+RZ+CX ring, 720 gates, P=480, H = sum ZZ + 0.5 sum X"}
    if not shift:
        return out
    hp = nat.Handle(20, device, nat.SVB_FP64)
    nshift = 48
    t0 = time.perf_counter()
    for p in range(nshift):
        for sgn in (1, -1):
            pp = pc.params.copy()
            pp[p] += sgn * math.pi / 2
            hp.reset()
            hp.set_circuit(pc.evaluated(pp))
            hp.run()
            hp.expectation(terms)
    t_shift = (time.perf_counter() - t0) / nshift * 480
    out.update({"param_shift_grads_per_s": 1.0 / t_shift, "speedup_vs_param_shift": t_shift / t_adj,
                "param_shift_sample": f"{nshift} of 480 parameters timed, scaled"})
    return out


def secondary_forms(device, circuit):
    """The other forms of the metric: per-gate FP64 sweeps and the fused FP32 tensor-core
    engine on the same circuit, the n=16 CPU-runnable case, batched QAOA, capacity,
    adjoint gradients (n=20, 480 params) and density matrices."""
    import torch
    from svsim_b200 import circuits, _native as nat
    forms = {}
    forms["per_gate_fp64"] = per_gate_form(device, circuit)
    forms["config1_n16_brickwork"] = config1_form(device)
    for k in (4, 5, 6):
        forms[f"fused_tc_fp32_k{k}"] = fused_form(device, circuit, k=k)
    forms["qaoa_batch_fp64"] = qaoa_form(device, 512, "fp64")
    forms["qaoa_batch_fp32"] = qaoa_form(device, 512, "fp32")
    forms["capacity"] = capacity_form(device)
    forms["adjoint"] = adjoint_form(device)
    forms["autotune"] = tuning_form(device)
    forms["reference_gpu_kernel"] = reference_gpu_form(device)
    forms["batched_circuits"] = batch_form(device)
    forms["density_matrix"] = density_form(device)
    return forms


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.form != "headline":
        run_form(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
