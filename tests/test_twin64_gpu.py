"""Errors of the f32 engine stated against its FP64 twin: the engine's own
direct convolution + growth, flow and gather functions instantiated in double
(flp_twin64_step, twin64.cu).

First the twin is tied to the FP64 oracle (the reference's algorithm restated
in double): both are double builds of the same statements, so they agree to
double rounding (their convolutions differ in algorithm only: direct here, FFT
in the oracle).  Then, at the blob 256x256 and multispecies 512x512 workloads,
one f32 engine step is taken from each state A_t of the f32 oracle trajectory
and compared with the twin's step from the same A_t, beside the f32 oracle's
own distance to the twin.
"""
import json
import os

import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import _native as nat
from autoverse_b200 import workloads as wl
from oracle import oracle as O

pytestmark = pytest.mark.gpu

THREADS = max(1, os.cpu_count() or 1)
TWIN_VS_ORACLE64 = 1e-10  # double builds of the same arithmetic


def twin_step(cfg, state):
    """(affinity, next state) of one FP64 twin step from `state`."""
    C = cfg["channels"]
    a = np.ascontiguousarray(state, dtype=np.float64).reshape(C, -1)
    aff = np.zeros_like(a)
    nxt = np.zeros_like(a)
    nat.check(nat.lib().flp_twin64_step(json.dumps(cfg).encode(), a.ctypes.data, aff.ctypes.data, nxt.ctypes.data))
    return aff, nxt


@pytest.mark.parametrize("case", ["blob64", "species96x64", "species_s075"])
def test_twin_equals_fp64_oracle(case):
    if case == "blob64":
        cfg, sd = wl.single_blob(64, R=9, blob_radius=0.15)
        st = O.seed_generate(sd, cfg)
    elif case == "species96x64":
        cfg, st = wl.multispecies(96, channels=2, R=9, patches=6, patch=16, seed=31, height=64)
    else:
        cfg, st = wl.multispecies(64, channels=2, R=7, patches=5, patch=12, seed=32)
        cfg["flow"]["distribution_size"] = 0.75
    o64 = O.OraclePropagator(cfg, f64=True)
    a64 = st.astype(np.float64).reshape(cfg["channels"], -1)
    for _ in range(3):
        aff, nxt = twin_step(cfg, a64)
        ref_aff = o64.affinity(a64)
        ref = o64.run(a64, 1, threads=THREADS)
        assert np.abs(aff - ref_aff).max() <= TWIN_VS_ORACLE64, np.abs(aff - ref_aff).max()
        assert np.abs(nxt - ref).max() <= TWIN_VS_ORACLE64, np.abs(nxt - ref).max()
        a64 = ref


def _errors_against_twin(cfg, st, steps, mode):
    """Per step t: max |engine(A_t) - twin(A_t)| and max |f32 oracle(A_t) - twin(A_t)|."""
    orc = O.OraclePropagator(cfg)
    a = np.ascontiguousarray(st, dtype=np.float32).reshape(cfg["channels"], -1)
    e_eng, e_orc = [], []
    with fl.CudaPropagator(cfg, conv_mode=mode) as p:
        for _ in range(steps):
            _, exact = twin_step(cfg, a)
            p.write_state(a)
            p.run_device(1)
            got = p.read_state().reshape(a.shape)
            nxt = orc.run(a, 1, threads=THREADS)
            e_eng.append(float(np.abs(got - exact).max()))
            e_orc.append(float(np.abs(nxt - exact).max()))
            a = nxt
    return np.array(e_eng), np.array(e_orc)


@pytest.mark.parametrize("mode", [fl.CONV_DIRECT, fl.CONV_FFT])
@pytest.mark.parametrize("workload", ["blob256", "multispecies512"])
def test_engine_error_against_its_fp64_twin(workload, mode):
    """The f32 engine's distance to the FP64 twin is the f32 rounding of the
    step: no larger than the f32 oracle's own distance to it, up to a small
    margin (the two round the convolution differently)."""
    if workload == "blob256":
        cfg, sd = wl.single_blob(256, R=13, blob_radius=0.1)
        st = O.seed_generate(sd, cfg)
    else:
        cfg, st = wl.multispecies(512, channels=3, R=15)
    e_eng, e_orc = _errors_against_twin(cfg, st, 20, mode)
    print(f"{workload} mode {mode}: engine vs FP64 twin per step max {e_eng.max():.3e} (median "
          f"{np.median(e_eng):.3e}); f32 oracle vs FP64 twin max {e_orc.max():.3e} (median {np.median(e_orc):.3e})")
    assert e_eng.max() <= 1.5 * e_orc.max() + 2e-6, (e_eng.max(), e_orc.max())
    assert e_eng.max() <= 5e-5
