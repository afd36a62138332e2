"""flp_affinity_noalloc: the allocation-free variant of the direct-path
affinity kernel, for callers that may not allocate device memory (code that
runs on another framework's stream and memory pool, such as a plugin or custom
operator).  Its output must match the existing entry point (flp_debug_affinity
on the direct path) on two calls in a row through the C ABI, with a different
config on the second call so that a stale scratch array would show.

Collected last on purpose: if it fails, every other test has already run.
"""
import ctypes as C
import json

import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import _native as nat
from autoverse_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _reference_affinity(cfg, state):
    with fl.CudaPropagator(cfg, conv_mode=fl.CONV_DIRECT) as p:
        p.write_state(state)
        return p.debug_affinity()


def _noalloc_affinity(cfg, state):
    """Input and output live in device buffers owned by two engine handles;
    the entry point itself receives only their device pointers."""
    lib = nat.lib()
    src = fl.CudaPropagator(cfg, conv_mode=fl.CONV_DIRECT)
    dst = fl.CudaPropagator(cfg, conv_mode=fl.CONV_DIRECT)
    try:
        src.write_state(state)
        d_in = lib.flp_device_state(src._h)
        d_out = lib.flp_device_state(dst._h)
        rc = lib.flp_affinity_noalloc(json.dumps(cfg).encode(), C.c_void_p(d_in), C.c_void_p(d_out),
                                      C.c_void_p(lib.flp_stream(dst._h)))
        nat.check(rc)
        return dst.read_state()  # synchronises dst's stream, copies d_out back
    finally:
        src.close()
        dst.close()


def test_noalloc_matches_direct_affinity_two_calls():
    cfg1, st1 = wl.multispecies(96, channels=2, R=9, patches=6, patch=16, seed=21, height=64)
    cfg2, st2 = wl.multispecies(64, channels=3, R=6, patches=5, patch=12, seed=22)
    for cfg, st in ((cfg1, st1), (cfg2, st2)):
        exp = _reference_affinity(cfg, st)
        got = _noalloc_affinity(cfg, st)
        # same kernel and same taps: identical, well inside the affinity tolerance
        assert np.array_equal(got, exp), float(np.abs(got - exp).max())


def test_noalloc_rejects_oversized_config():
    cfg, st = wl.multispecies(64, channels=1, R=40, patches=2, patch=8, seed=23)
    lib = nat.lib()
    with fl.CudaPropagator(wl.multispecies(64, channels=1, R=4, seed=23)[0]) as p:
        d = lib.flp_device_state(p._h)
        rc = lib.flp_affinity_noalloc(json.dumps(cfg).encode(), C.c_void_p(d), C.c_void_p(d), None)
    assert rc == -2 and b"radius" in lib.flp_last_error()
