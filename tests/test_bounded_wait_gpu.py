"""Bounded device waits, run through the C-ABI (gpudb_compile + gpudb_execute).

Every spin-wait in the engine's kernels (mbarrier waits of the TMA scan
ring, flag waits) gives up after GPUDB_WAIT_NS of %globaltimer time, sets
GPUDB_DEVERR_WAIT_TIMEOUT in the device error word and returns, so a wait
that can never finish ends the kernel with an error status instead of
hanging the GPU. This test makes such a wait run out on purpose, in the
safe way: one CTA waits on an mbarrier that nothing arrives at, with the
bound lowered to 1 ms at compile time and no bulk copy in flight in that
CTA. The call must return GPUDB_E_DEVICE with the timeout bit, and the
same context must run the next query correctly.
"""
import ctypes as C
from pathlib import Path

import pytest

from gpudbmetalcodegen_b200 import _lib
from gpudbmetalcodegen_b200 import workloads as W
from oracle import oracle_py as O

pytestmark = pytest.mark.gpu
GPUDB_E_DEVICE = -7  # include/gpudb_rt.h: a kernel reported a device error word

HEADER = Path(__file__).resolve().parent.parent / "gpudbmetalcodegen_b200" / "csrc" / "kernels" / "gpudb_device.cuh"

KERNEL = r"""
// one CTA: thread 0 initialises an mbarrier expecting one arrival, and no
// thread ever arrives; every thread's wait gives up after GPUDB_WAIT_NS
extern "C" __global__ void wait_for_nothing(unsigned* __restrict__ gpudb_err, unsigned long long* __restrict__ gave_up) {
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) {
        gpudb_mbar_init(&bar, 1u);
        gpudb_mbar_init_fence();
    }
    __syncthreads();
    const unsigned long long t0 = gpudb_now_ns();
    if (!gpudb_mbar_wait(&bar, 0u, gpudb_err)) atomicAdd(gave_up, 1ull);
    if (threadIdx.x == 0) atomicMax(gave_up + 1, gpudb_now_ns() - t0);
}
"""


def _run_waiting_kernel(ctx):
    lib = _lib.load()
    src = "#define GPUDB_WAIT_NS 1000000ull  // 1 ms\n" + HEADER.read_text() + KERNEL
    mod = C.c_void_p()
    names = (C.c_char_p * 1)(b"wait_for_nothing")
    _lib.check(lib.gpudb_compile(ctx.handle, src.encode(), names, 1, C.byref(mod)), ctx.handle)
    binds = (_lib.BindingDesc * 2)(
        _lib.BindingDesc(b"gpudb_err", _lib.PARAM_ERROR_WORD, b"unsigned", None, None, 1, 0, 0),
        _lib.BindingDesc(b"wt_gave_up", _lib.PARAM_DEVICE_BUFFER, b"unsigned long long", None, b"2", 1, 0, 0))
    phase = (_lib.PhaseDesc * 1)(_lib.PhaseDesc(b"wait_for_nothing", None, 64, 1, 0, 0, 0, 1, binds, 2))
    t = _lib.Timing()
    st = lib.gpudb_execute(ctx.handle, mod, phase, 1, 0, 1, 0, 1, C.byref(t))
    out = (C.c_uint64 * 2)()
    _lib.check(lib.gpudb_read_buffer(ctx.handle, b"wt_gave_up", out, 16), ctx.handle)
    lib.gpudb_module_free(mod)
    return st, t.device_error, int(out[0]), int(out[1])


def test_wait_that_never_completes_times_out_and_the_context_stays_usable(ctx):
    st, err, gave_up, waited_ns = _run_waiting_kernel(ctx)
    assert st == GPUDB_E_DEVICE, _lib.last_error(ctx.handle)
    assert err & 0x2, err  # GPUDB_DEVERR_WAIT_TIMEOUT
    assert gave_up == 64  # every thread of the CTA gave up and returned
    assert 1_000_000 <= waited_ns < 1_000_000_000, waited_ns  # after the 1 ms bound, well before the default 1 s
    # the same context runs the next query correctly
    f = W.gen_fact(50_000, seed=4)
    ctx.upload_table("fact", f)
    res, t = ctx.run("template=q1")
    assert t.device_error == 0
    got, expect = res.as_dicts(), O.q1(f)
    assert [(g["flag_a"], g["flag_b"]) for g in got] == [(e["flag_a"], e["flag_b"]) for e in expect]
    for g, e in zip(got, expect):
        for k in O.Q1_AGGS:
            assert g[k] == e[k], k
    # and the timeout repeats identically (the error word was cleared)
    st2, err2, gave_up2, _ = _run_waiting_kernel(ctx)
    assert (st2, err2 & 0x2, gave_up2) == (st, 0x2, 64)
