"""B200-native runtime-codegen backend for a GPUDBMetalCodeGen-style engine.

Plans (scan / filter / join / group-by / top-k pipelines) are lowered to
fused CUDA C++ by the operator emitters in ``csrc/``, compiled at run time
by NVRTC for sm_100a and launched through the C-ABI of ``lib/libgpudb.so``
(include/gpudb_rt.h, include/gpudb_engine.h). This package is the Python
host mirror of that API.
"""
from .engine import Context, Query, Result, Timing, compare_canonical, compile_check, templates  # noqa: F401

# Plans compiled ahead of time into the in-tree cubin cache by prewarm().
STANDARD_PLANS = [
    ("template=q1", ""), ("template=q1", "scan=direct"), ("template=q6", ""), ("template=q6", "scan=direct"),
    ("template=join_topk", ""), ("template=join_topk", "scan=direct"), ("template=join_rows", ""),
    ("template=groupby", ""), ("template=groupby", "smem=11"), ("template=groupby", "layout=bucket8"),
    ("template=hashjoin", ""), ("template=hashjoin", "smem=11"),
    ("template=colmax;table=dim;col=b_key", "bs=512;scan=direct"),
    ("template=colmax;table=mixdim;col=md_key", "bs=512;scan=direct"),
]


def prewarm_kernel_cache(plans=None) -> int:
    """NVRTC-compile plans for sm_100a into the cubin cache (no GPU needed)."""
    n = 0
    for spec, tune in plans or STANDARD_PLANS:
        Query(spec, tune).close()
        n += 1
    return n
