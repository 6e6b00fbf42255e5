"""Build the reference pinning harness into oracle/_ref/ — TEST INFRASTRUCTURE.

1. Compiles the reference engine's planning / operator / codegen sources
   exactly as they lie in the reference tree (no copies) together with
   ref_msl_driver.cpp into oracle/_ref/ref_msl_driver.
2. Runs it: the reference generates the MSL kernels of the benchmark
   pipelines (oracle/_ref/ref_<plan>.cpp + manifest.json).
3. Compiles those kernels as C++ against msl_cpu_shim.h into
   oracle/_ref/libref_kernels.so, loaded by oracle/ref_harness/ref_run.py.

Needs the reference source tree: the directory named by the environment
variable GPUDB_REFERENCE_ROOT, by default /root/reference (present in the
build container, not on GPU hosts); oracle/_ref/ is git-ignored.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
REF = Path(os.environ.get("GPUDB_REFERENCE_ROOT", "/root/reference"))

REF_SOURCES = [
    "codegen/planning/metal_plan_builder.cpp",
    "codegen/operators/metal_operators.cpp",
    "codegen/core/metal_codegen_base.cpp",
    "codegen/core/metal_param_binding.cpp",
]
REF_INCLUDES = ["codegen/planning", "codegen/operators", "codegen/core"]
PLANS = ["Q1", "Q6", "JOIN", "JOINROWS", "GROUPBY", "ANTI", "HIST", "DIRECT", "Q5"]


def available() -> bool:
    """True when the reference source tree is present on this host."""
    return all((REF / s).is_file() for s in REF_SOURCES)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference harness build step failed:\n" + " ".join(map(str, cmd)) + "\n" + r.stdout +
                           r.stderr[-4000:])
    return r.stdout


def build(force: bool = False) -> Path:
    if not available():
        raise RuntimeError(f"the reference tree is not available on this host ({REF}; set GPUDB_REFERENCE_ROOT)")
    OUT.mkdir(exist_ok=True)
    lib = OUT / "libref_kernels.so"
    inputs = [HERE / "ref_msl_driver.cpp", HERE / "msl_cpu_shim.h", Path(__file__)] + [REF / s for s in REF_SOURCES]
    if not force and lib.exists() and lib.stat().st_mtime >= max(p.stat().st_mtime for p in inputs):
        return lib
    driver = OUT / "ref_msl_driver"
    _run(["g++", "-std=c++20", "-O1", "-w", *[f"-I{REF / d}" for d in REF_INCLUDES], str(HERE / "ref_msl_driver.cpp"),
          *[str(REF / s) for s in REF_SOURCES], "-o", str(driver)])
    _run([str(driver), str(OUT)])
    _run(["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-w", "-Wno-attributes", f"-I{HERE}",
          *[str(OUT / f"ref_{p}.cpp") for p in PLANS], "-o", str(lib), "-lpthread"])
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
