"""Build the CPU oracle (oracle/liboracle.so) — test infrastructure only.

gcc -O3 -fopenmp; portable x86-64-v2 code so the library built here also
runs on the GPU box's host CPU.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


def build(force: bool = False) -> Path:
    src = HERE / "oracle.c"
    hdr = HERE / "oracle.h"
    if not force and LIB.exists() and LIB.stat().st_mtime >= max(src.stat().st_mtime, hdr.stat().st_mtime):
        return LIB
    # built under a per-process name and renamed into place, so processes
    # that build at the same time (replicas) never load a half-written file
    tmp = LIB.with_name(f"liboracle.{os.getpid()}.so")
    cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", "-std=gnu11", "-Wall", "-Wextra",
           "-o", str(tmp), str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
