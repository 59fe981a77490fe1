"""TEST INFRASTRUCTURE: builds tests/native/_build/libstaged_emu.so — the CPU runner of
staged plans (staged_emulator.cu) linked with the product's planner and lowering."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CSRC = os.path.join(ROOT, "sv-sim_b200", "csrc")
OUT = os.path.join(HERE, "_build", "libstaged_emu.so")


def build() -> str:
    srcs = [os.path.join(HERE, "staged_emulator.cu"), os.path.join(CSRC, "plan.cpp"),
            os.path.join(CSRC, "lower.cpp"), os.path.join(CSRC, "fuse.cpp"), os.path.join(CSRC, "pairs.cpp")]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    if os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(d) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
           "-o", OUT] + srcs
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(), file=sys.stderr)
