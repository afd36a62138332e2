"""Failure detection on the GPU, in forms that fault, trap or hang no GPU.

* Non-finite state: a NaN or an infinity written into a host state is caught
  by the flow pass's bound check and reported by the next synchronize as
  FLP_ERR_NONFINITE (single world, batched worlds, parameter-embedded
  world), the handle stays usable afterwards (the reference has no such
  check: its NaNs propagate silently, src/compute/propagator.rs:239-420).
* Bounded host waits: flp_synchronize_for / flp_batch_synchronize_for give up
  with FLP_ERR_TIMEOUT while work is still queued, cancel nothing, and a
  plain synchronize afterwards succeeds.
* Out of device memory: the library's allocation hook makes the n-th device
  allocation fail (on the host, the driver is not called); every create
  entry point must return FLP_ERR_OOM for each n and give back everything it
  had allocated (live allocation count back to its baseline).
The worlds with a non-finite state are small (at most 96 cells a side): a
non-finite displacement widens the gather window to the torus-covering
bound, which the general gather path walks cell by cell.
"""
import ctypes as C
import json

import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import _native as nat
from autoverse_b200 import workloads as wl

pytestmark = pytest.mark.gpu

NONFINITE, TIMEOUT, OOM = -6, -5, -3


def _code(excinfo):
    return excinfo.value.code


@pytest.mark.parametrize("bad", [np.nan, np.inf])
@pytest.mark.parametrize("mode", [fl.CONV_DIRECT, fl.CONV_FFT])
def test_nonfinite_single_world(bad, mode):
    cfg, st = wl.multispecies(64, channels=2, R=6, patches=4, patch=16, seed=31)
    poisoned = st.copy()
    poisoned[1, 40 * 64 + 17] = bad
    with fl.CudaPropagator(cfg, conv_mode=mode) as p:
        p.write_state(poisoned)
        p.run_device(1)
        with pytest.raises(fl.FlpError) as e:
            p.synchronize()
        assert _code(e) == NONFINITE
        # reported once; the handle keeps working on a clean state
        p.write_state(st)
        p.run_device(3)
        p.synchronize()
        got = p.read_state()
    with fl.CudaPropagator(cfg, conv_mode=mode) as q:
        q.write_state(st)
        q.run_device(3)
        assert np.array_equal(got, q.read_state())


def test_nonfinite_batched_world():
    worlds = wl.batched_worlds(3, sides=(64, 96), seed=32)
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        b.load_seeds([s for _, s in worlds])
        clean = b.read_world(1)
        poisoned = clean.copy()
        poisoned[0, poisoned.shape[1] // 2] = np.nan
        b.write_world(1, poisoned)
        b.run(1)
        with pytest.raises(fl.FlpError) as e:
            b.synchronize()
        assert _code(e) == NONFINITE
        b.write_world(1, clean)
        b.run(2)
        b.synchronize()
        assert np.isfinite(b.read_world(1)).all()


def test_nonfinite_embedded_world():
    rng = np.random.default_rng(33)
    cfg = wl.config(48, 32, 1, [wl.kernel(rings=wl.random_rings(rng))], kernel_radius=6)
    cfg["embedding"] = {"enabled": True, "mixing_temperature": 1.0, "linear_mixing": False}
    st = np.zeros((1, 48 * 32), np.float32)
    st[0, 10 * 48 + 10: 10 * 48 + 22] = rng.random(12, dtype=np.float32)
    params = np.tile(np.float32([0.15, 0.015, 1.0, 1.0, 2.0]), (1, 48 * 32, 1))
    poisoned = st.copy()
    poisoned[0, 10 * 48 + 12] = np.nan
    with fl.EmbeddedPropagator(cfg) as p:
        p.write(fl.EmbeddedState(poisoned, params, 48, 32))
        p.run_device(1)
        with pytest.raises(fl.FlpError) as e:
            p.synchronize()
        assert _code(e) == NONFINITE
        p.write(fl.EmbeddedState(st, params, 48, 32))
        p.run_device(2)
        p.synchronize()


def test_bounded_wait_single_world():
    cfg, st = wl.multispecies(512, channels=3, R=15)
    with fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p:
        p.write_state(st)
        p.synchronize()
        p.run_device(2000)  # about 0.1 s of device work
        with pytest.raises(fl.FlpError) as e:
            p.synchronize(timeout_ms=1.0)
        assert _code(e) == TIMEOUT
        p.synchronize()  # the queued steps were not cancelled
        assert p.info().step == 2000
        p.synchronize(timeout_ms=1000.0)  # nothing pending: returns at once


def test_bounded_wait_batch():
    worlds = wl.batched_worlds(64, sides=(128, 256), seed=34)
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        b.load_seeds([s for _, s in worlds])
        b.synchronize()
        b.run(400)
        with pytest.raises(fl.FlpError) as e:
            b.synchronize(timeout_ms=0.5)
        assert _code(e) == TIMEOUT
        b.synchronize()


# ---- out of device memory -------------------------------------------------

def _live():
    v = C.c_int64()
    nat.check(nat.lib().flp_debug_live_device_allocs(C.byref(v)))
    return v.value


def _strings(items):
    enc = [json.dumps(c).encode() for c in items]
    return (C.c_char_p * len(enc))(*enc), enc


def _oom_sweep(create, destroy, limit=2000):
    """create() -> (rc, handle).  Fails the n-th allocation for n = 0, 1, ...
    until a create succeeds; every failing create must return OOM and leave
    the live allocation count where it was."""
    lib = nat.lib()
    rc, h = create()  # first create: process-wide caches (twiddles, tuning) settle
    nat.check(rc)
    destroy(h)
    base = _live()
    failures = 0
    try:
        for n in range(limit):
            lib.flp_debug_fail_device_alloc(n)
            rc, h = create()
            if rc == 0:
                lib.flp_debug_fail_device_alloc(-1)
                destroy(h)
                break
            assert rc == OOM, (n, rc, lib.flp_last_error())
            assert _live() == base, (n, _live(), base)
            failures += 1
        else:
            pytest.fail("create never succeeded")
    finally:
        lib.flp_debug_fail_device_alloc(-1)
    assert failures > 0
    assert _live() == base
    return failures


def test_oom_single_world_create():
    lib = nat.lib()
    for cfg in (wl.multispecies(64, channels=2, R=6, seed=35)[0], wl.sphere3d(32, R=5)[0]):
        js = json.dumps(cfg).encode()

        def create():
            h = C.c_void_p()
            return lib.flp_create(js, C.byref(h)), h

        n = _oom_sweep(create, lambda h: lib.flp_destroy(h))
        assert n >= 5


def test_oom_batch_create():
    lib = nat.lib()
    arr, keep = _strings([c for c, _ in wl.batched_worlds(4, sides=(64, 128), seed=36)])

    def create():
        h = C.c_void_p()
        return lib.flp_batch_create(arr, len(keep), C.byref(h)), h

    assert _oom_sweep(create, lambda h: lib.flp_batch_destroy(h)) >= 5


def test_oom_embedded_and_adjoint_create():
    lib = nat.lib()
    rng = np.random.default_rng(37)
    ce = wl.config(48, 32, 1, [wl.kernel(rings=wl.random_rings(rng))], kernel_radius=6)
    ce["embedding"] = {"enabled": True, "mixing_temperature": 1.0, "linear_mixing": False}
    js = json.dumps(ce).encode()

    def create_emb():
        h = C.c_void_p()
        return lib.flp_emb_create(js, C.byref(h)), h

    assert _oom_sweep(create_emb, lambda h: lib.flp_emb_destroy(h)) >= 3
    arr, keep = _strings([c for c, _ in wl.adjoint_worlds(2, size=64, R=8, seed=38)])

    def create_adj():
        h = C.c_void_p()
        return lib.flp_adj_create(arr, len(keep), C.byref(h)), h

    assert _oom_sweep(create_adj, lambda h: lib.flp_adj_destroy(h)) >= 3
