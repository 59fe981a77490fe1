"""Build of the native library libsvsim_b200.so (sm_100a) with nvcc.

Sources live in sv-sim_b200/csrc, objects in sv-sim_b200/_build, and the library is
written in-tree to sv-sim_b200/svsim_b200/lib/ so it travels with the working tree.
nvcc cross-compiles for sm_100a without a GPU present.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
PROJECT = os.path.dirname(PKG_DIR)                  # sv-sim_b200/
ROOT = os.path.dirname(PROJECT)                     # repository root
CSRC = os.path.join(PROJECT, "csrc")
OBJ_DIR = os.path.join(PROJECT, "_build")
LIB_DIR = os.path.join(PKG_DIR, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libsvsim_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                     "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]


# Per-source extra flags.  The per-gate engine keeps every rounding of the reference's
# CPU arithmetic (no fused multiply-add), so its FP64 states are bit-identical to it.
EXTRA_FLAGS = {"kernels_pergate.cu": ["-fmad=false"]}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cpp")))


def headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    newest = max([_mtime(src)] + [_mtime(h) for h in headers()])
    if _mtime(obj) >= newest:
        return obj
    cmd = [nvcc()] + NVCC_FLAGS + EXTRA_FLAGS.get(os.path.basename(src), []) + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
    if res.stderr.strip() and verbose:
        print(res.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    if force:
        for f in os.listdir(OBJ_DIR):
            os.remove(os.path.join(OBJ_DIR, f))
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _mtime(LIB_PATH) < max(_mtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB_PATH] + objs + ["-lcudart_static", "-lrt",
                                                                      "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB_PATH


def ptxas_report(src_name: str) -> str:
    """Register / shared-memory usage of one source (nvcc -Xptxas -v)."""
    src = os.path.join(CSRC, src_name)
    cmd = [nvcc()] + NVCC_FLAGS + EXTRA_FLAGS.get(src_name, []) + ["-Xptxas", "-v", "-c", src, "-o", os.devnull]
    res = subprocess.run(cmd, capture_output=True, text=True)
    return res.stdout + res.stderr


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
