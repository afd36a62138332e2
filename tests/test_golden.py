"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py
from the CPU oracle): reduced-size instances of the single-blob, multispecies,
batched-world and 3D-sphere configurations with their initial state, first
affinity and flow, and the states after 1 and 10 steps.

CPU tests: the oracle still reproduces every fixture bit for bit (so a change
to the restatement cannot slip through).  GPU tests: the engine's transport
stage, fed the fixture's state and affinity, reproduces step1 bit for bit;
full steps stay within 1e-5 (1 step) and 1e-4 (10 steps); batched worlds the same.
"""
import glob
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
NAMES = [os.path.basename(p)[:-4] for p in GOLDEN]


def load(name):
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    return json.loads(str(z["config"])), {k: z[k] for k in z.files if k != "config"}


def test_fixtures_present():
    assert {"blob64_R13", "multispecies64x48_C3_R15", "sphere32_R10"} <= set(NAMES)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name):
    cfg, g = load(name)
    orc = O.OraclePropagator(cfg)
    np.testing.assert_array_equal(orc.affinity(g["state0"]), g["aff0"])
    s1 = orc.run(g["state0"], 1)
    np.testing.assert_array_equal(s1, g["step1"])
    np.testing.assert_array_equal(orc.last_flow(), g["flow0"])
    np.testing.assert_array_equal(orc.run(s1, 9), g["step10"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_engine_against_golden(name):
    import autoverse_b200 as fl
    cfg, g = load(name)
    with fl.CudaPropagator(cfg) as p:
        got = p.debug_transport(g["state0"], g["aff0"])
        assert np.array_equal(got, g["step1"]), np.abs(got - g["step1"]).max()
        p.write_state(g["state0"])
        p.run_device(1)
        assert np.abs(p.read_state() - g["step1"]).max() <= 1e-5
        p.run_device(9)
        assert np.abs(p.read_state() - g["step10"]).max() <= 1e-4


@pytest.mark.gpu
def test_batched_against_golden():
    import autoverse_b200 as fl
    names = [n for n in NAMES if n.startswith("batch_world")]
    loaded = [load(n) for n in names]
    with fl.BatchedPropagator([c for c, _ in loaded]) as b:
        for i, (_, g) in enumerate(loaded):
            b.write_world(i, g["state0"])
        b.run(1)
        for i, (_, g) in enumerate(loaded):
            assert np.abs(b.read_world(i) - g["step1"]).max() <= 1e-5, names[i]
        b.run(9)
        for i, (_, g) in enumerate(loaded):
            assert np.abs(b.read_world(i) - g["step10"]).max() <= 1e-4, names[i]
