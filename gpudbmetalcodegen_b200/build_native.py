"""Build libgpudb.so in-tree (gpudbmetalcodegen_b200/lib/).

Host C++ is compiled with g++, CUDA sources with nvcc for sm_100a
(-gencode arch=compute_100a,code=sm_100a). Generated query kernels are not
compiled here: the runtime compiles them with NVRTC for sm_100a at run time
(``prewarm_kernel_cache`` can compile the standard plans ahead of time into
the in-tree cubin cache, which needs no GPU).

Usage: python -m gpudbmetalcodegen_b200.build_native [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "lib"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O2", "-g", "-fPIC", "-std=c++17", "-Wall", "-Wextra", "-Wno-unused-parameter",
            f"-I{CUDA_HOME / 'include'}", f"-I{INCLUDE}"]
NVCCFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
             f"-I{INCLUDE}", f"-I{CSRC / 'kernels'}"] + ARCH

HOST_SOURCES = [
    "core/param_binding.cpp",
    "core/cuda_codegen.cpp",
    "operators/cuda_operators.cpp",
    "planning/plan_builder.cpp",
    "planning/query_ir.cpp",
    "execution/cuda_api.cpp",
    "execution/runtime_compiler.cpp",
    "execution/result_collector.cpp",
    "execution/executor.cpp",
    "execution/query_engine.cpp",
    "capi/gpudb_capi.cpp",
    "io/colbin.cpp",
    "sql/sql_frontend.cpp",
]
CUDA_SOURCES: list[str] = [
    "kernels/noalloc_distinct.cu",
    "kernels/sizer_mlp.cu",
    "kernels/batch_kernels.cu",
]

LIB_NAME = "libgpudb.so"
# the seeded synthetic-table generators: their own library, so that data
# generation (CPU baselines, fixtures) maps no engine code
DATAGEN_HOST_SOURCES = ["datagen/datagen.cpp"]
DATAGEN_CUDA_SOURCES = ["kernels/datagen_device.cu"]
DATAGEN_LIB_NAME = "libgpudb_datagen.so"


def _headers() -> list[Path]:
    hs = list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.cuh")) + list(CSRC.rglob("*.inc")) + list(INCLUDE.glob("*.h"))
    return [h for h in hs if h.is_file()]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], log: list[str]) -> None:
    log.append(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.stdout.strip():
        log.append(r.stdout.strip())
    if r.stderr.strip():
        log.append(r.stderr.strip())
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def embed_device_header() -> Path:
    """Embed gpudb_device.cuh as a C++ string literal (device_header_gen.inc)."""
    src = CSRC / "kernels" / "gpudb_device.cuh"
    out = CSRC / "core" / "device_header_gen.inc"
    if not _stale(out, [src]):
        return out
    text = src.read_text()
    parts = []
    # raw-string chunks keep each literal well below compiler limits
    step = 8000
    for i in range(0, len(text), step):
        parts.append('R"GPUDBHDR(' + text[i:i + step] + ')GPUDBHDR"')
    out.write_text("// generated from kernels/gpudb_device.cuh by build_native.py; do not edit\n" + "\n".join(parts) + "\n")
    return out


def _build_lib(name: str, host: list[str], cuda: list[str], extra: list[str], headers: list[Path], force: bool,
               log: list[str]) -> Path:
    objs = []
    for rel in host:
        src = CSRC / rel
        obj = BUILD / (rel.replace("/", "_") + ".o")
        if force or _stale(obj, [src] + headers):
            _run([CXX, *CXXFLAGS, "-c", str(src), "-o", str(obj)], log)
        objs.append(obj)
    for rel in cuda:
        src = CSRC / rel
        obj = BUILD / (rel.replace("/", "_") + ".o")
        if force or _stale(obj, [src] + headers):
            _run([NVCC, *NVCCFLAGS, "-c", str(src), "-o", str(obj)], log)
        objs.append(obj)
    lib = LIB / name
    if force or _stale(lib, objs):
        cudalib = CUDA_HOME / "lib64"
        _run([NVCC, "-shared", *ARCH, "-o", str(lib), *map(str, objs),
              f"-L{cudalib}", *extra, "-cudart", "static", "-ldl", "-lpthread", "-lrt",
              f"-Xlinker", f"-rpath={cudalib}"], log)
    return lib


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    embed_device_header()
    headers = _headers()
    log: list[str] = []
    lib = _build_lib(LIB_NAME, HOST_SOURCES, CUDA_SOURCES, ["-lnvrtc"], headers, force, log)
    _build_lib(DATAGEN_LIB_NAME, DATAGEN_HOST_SOURCES, DATAGEN_CUDA_SOURCES, [], headers, force, log)
    if verbose:
        print("\n".join(log))
    return lib


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose=True)
    print(p)
