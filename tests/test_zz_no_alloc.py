"""flp_affinity_noalloc: the allocation-free variant of the direct-path
affinity kernel, for callers that may not allocate device memory (code that
runs on another framework's stream and memory pool, such as a plugin or custom
operator).  Its output must match the existing entry point (flp_debug_affinity
on the direct path) on two calls in a row through the C ABI, with a different
config on the second call so that a stale scratch array would show; it must
stay within the affinity tolerance of the FP64 oracle; and the device's free
memory must not change across calls.

Collected last on purpose: if it fails, every other test has already run.
"""
import ctypes as C
import json

import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import _native as nat
from autoverse_b200 import workloads as wl
from oracle import oracle as O

pytestmark = pytest.mark.gpu

AFF_FACTOR = 4.0  # the affinity tolerance of the parity suite
AFF_ABS = 2e-6


def _reference_affinity(cfg, state):
    with fl.CudaPropagator(cfg, conv_mode=fl.CONV_DIRECT) as p:
        p.write_state(state)
        return p.debug_affinity()


class _Buffers:
    """Input and output device buffers owned by two engine handles; the entry
    point itself receives only their device pointers."""

    def __init__(self, cfg, state):
        self.cfg = cfg
        self.src = fl.CudaPropagator(cfg, conv_mode=fl.CONV_DIRECT)
        self.dst = fl.CudaPropagator(cfg, conv_mode=fl.CONV_DIRECT)
        self.src.write_state(state)
        self.src.synchronize()

    def call(self):
        lib = nat.lib()
        d_in = lib.flp_device_state(self.src._h)
        d_out = lib.flp_device_state(self.dst._h)
        rc = lib.flp_affinity_noalloc(json.dumps(self.cfg).encode(), C.c_void_p(d_in), C.c_void_p(d_out),
                                      C.c_void_p(lib.flp_stream(self.dst._h)))
        nat.check(rc)
        self.dst.synchronize()

    def result(self):
        return self.dst.read_state()  # copies the device output back

    def close(self):
        self.src.close()
        self.dst.close()


def _free_bytes():
    import torch
    return torch.cuda.mem_get_info(0)[0]


def test_noalloc_matches_direct_affinity_two_calls():
    cfg1, st1 = wl.multispecies(96, channels=2, R=9, patches=6, patch=16, seed=21, height=64)
    cfg2, st2 = wl.multispecies(64, channels=3, R=6, patches=5, patch=12, seed=22)
    cases = [(cfg1, st1), (cfg2, st2)]
    expected = [_reference_affinity(c, s) for c, s in cases]
    bufs = [_Buffers(c, s) for c, s in cases]
    try:
        # first calls: look up the scratch address, load the kernels
        for b in bufs:
            b.call()
        free0 = _free_bytes()
        # two calls in a row, different configs: each must rewrite the scratch
        for b, exp, (cfg, st) in zip(bufs, expected, cases):
            b.call()
            got = b.result()
            # same kernel and same taps: identical, well inside the affinity tolerance
            assert np.array_equal(got, exp), float(np.abs(got - exp).max())
            exp32 = O.OraclePropagator(cfg).affinity(st)
            exp64 = O.OraclePropagator(cfg, f64=True).affinity(st.astype(np.float64))
            err_orc = np.abs(exp32 - exp64).max()
            err = np.abs(got - exp64).max()
            assert err <= AFF_FACTOR * err_orc + AFF_ABS, (err, err_orc)
        assert _free_bytes() == free0, "device memory changed across allocation-free calls"
    finally:
        for b in bufs:
            b.close()


def test_noalloc_rejects_oversized_config():
    cfg, st = wl.multispecies(64, channels=1, R=40, patches=2, patch=8, seed=23)
    lib = nat.lib()
    with fl.CudaPropagator(wl.multispecies(64, channels=1, R=4, seed=23)[0]) as p:
        d = lib.flp_device_state(p._h)
        rc = lib.flp_affinity_noalloc(json.dumps(cfg).encode(), C.c_void_p(d), C.c_void_p(d), None)
    assert rc == -2 and b"radius" in lib.flp_last_error()
