"""Builds the reference's own front-end sources, unchanged, against the drop-in headers.

The drop-in (include/svsim_dropin/*) exposes the reference's class Simulation / Gate
API over libsvsim_b200.so.  To show that it is a drop-in, three unmodified reference
sources are compiled against it, straight from the reference tree (read from stdin;
nothing is copied into this repository):

  * svsim/src/py_wrapper.cpp                    -> lib/libsvsim<EXT_SUFFIX>  (module libsvsim)
  * svsim/unit_test/unit_test_nvgpu_sin.cu      -> lib/dropin_unit_test      (14 gate KATs)
  * svsim/example/adder_n10_nvgpu_sin.cu        -> lib/dropin_adder_n10      (Cuccaro adder)

They include their headers as "config.hpp" or "../src/svsim_nvgpu_sin.cuh"; compiling
from stdin inside a scratch directory whose ../src holds links to the drop-in headers
makes those quoted includes resolve to the drop-in.  The reference tree's location is
the caller's argument or the SVSIM_REFERENCE environment variable; when neither names an
existing tree (e.g. on a machine without the reference) the previously built artefacts
are used as they are.
"""
from __future__ import annotations

import os
import subprocess
import sysconfig

from .build import LIB_DIR, LIB_PATH, PROJECT, ROOT

DROPIN = os.path.join(ROOT, "include", "svsim_dropin")
SCRATCH = os.path.join(PROJECT, "_build", "dropin")
EXT = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
MODULE = os.path.join(LIB_DIR, "libsvsim" + EXT)
UNIT_TEST = os.path.join(LIB_DIR, "dropin_unit_test")
ADDER = os.path.join(LIB_DIR, "dropin_adder_n10")


def _scratch():
    """<SCRATCH>/src -> drop-in headers; <SCRATCH>/work is the compile directory."""
    src = os.path.join(SCRATCH, "src")
    work = os.path.join(SCRATCH, "work")
    os.makedirs(src, exist_ok=True)
    os.makedirs(work, exist_ok=True)
    for f in os.listdir(DROPIN):
        link = os.path.join(src, f)
        if not os.path.lexists(link):
            os.symlink(os.path.join(DROPIN, f), link)
        wlink = os.path.join(work, f)
        if not os.path.lexists(wlink):
            os.symlink(os.path.join(DROPIN, f), wlink)
    return work


def _compile_stdin(source: str, out: str, extra: list[str]):
    work = _scratch()
    cmd = ["g++", "-O3", "-std=c++17", "-x", "c++", "-", "-I" + DROPIN,
           "-I" + os.path.join(ROOT, "include"), "-o", out] + extra + [
        "-L" + LIB_DIR, "-lsvsim_b200", "-Wl,-rpath,$ORIGIN"]
    with open(source, "rb") as f:
        subprocess.run(cmd, stdin=f, cwd=work, check=True)


def build_python_module(force: bool = False, reference: str | None = None) -> str | None:
    """Builds the three reference front ends from the reference tree at `reference`
    (default: $SVSIM_REFERENCE) against the drop-in headers."""
    reference = reference or os.environ.get("SVSIM_REFERENCE", "")
    REF_SRC = os.path.join(reference, "svsim") if reference else ""
    if not REF_SRC or not os.path.isdir(REF_SRC):
        return MODULE if os.path.exists(MODULE) else None
    import pybind11
    srcs = {
        MODULE: (os.path.join(REF_SRC, "src", "py_wrapper.cpp"),
                 ["-shared", "-fPIC", "-DUSE_NVGPU", "-I" + pybind11.get_include(),
                  "-I" + sysconfig.get_paths()["include"]]),
        UNIT_TEST: (os.path.join(REF_SRC, "unit_test", "unit_test_nvgpu_sin.cu"), []),
        ADDER: (os.path.join(REF_SRC, "example", "adder_n10_nvgpu_sin.cu"), []),
    }
    headers = [os.path.join(DROPIN, f) for f in os.listdir(DROPIN)]
    for out, (src, extra) in srcs.items():
        deps = [src, LIB_PATH] + headers
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(
                os.path.getmtime(d) for d in deps):
            continue
        _compile_stdin(src, out, extra)
    return MODULE
