"""CPU-side checks of the engine: the C ABI library loads and exports every
symbol the public header declares, the host-side seed generator and config
validation agree with the oracle, and the CUDA path fails loudly (no CPU
fallback) when no device is present."""
import json

import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import _native as nat
from autoverse_b200 import workloads as wl
from oracle import oracle as O


def test_library_exports_header_symbols():
    lib = nat.lib()
    syms = nat.header_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/flowlenia_cuda.h but not exported"


SEEDS_2D = [
    {"pattern": {"type": "GaussianBlob", "center": [0.5, 0.5], "radius": 0.1, "amplitude": 1.0, "channel": 0}},
    {"pattern": {"type": "MultiBlob", "blobs": [
        {"center": [0.3, 0.5], "radius": 0.1, "amplitude": 1.0, "channel": 0},
        {"center": [0.7, 0.5], "radius": 0.1, "amplitude": 2.0, "channel": 1}]}},
    {"pattern": {"type": "Ring", "center": [0.4, 0.6], "inner_radius": 0.1, "outer_radius": 0.3, "amplitude": 0.8,
                 "channel": 1}},
    {"pattern": {"type": "Noise", "amplitude": 0.5, "channel": None, "seed": 42}},
    {"pattern": {"type": "Noise", "amplitude": 0.5, "channel": 1, "seed": 7}},
    {"pattern": {"type": "Custom", "values": [[0, 0, 0, 0.5], [5, 3, 1, 0.25], [99, 99, 0, 9.0]]}},
]

SEEDS_3D = [
    {"pattern": {"type": "GaussianSphere", "center": [0.5, 0.5, 0.5], "radius": 0.2, "amplitude": 1.0,
                 "channel": 0}},
    {"pattern": {"type": "MultiSphere", "spheres": [
        {"center": [0.3, 0.5, 0.5], "radius": 0.1, "amplitude": 1.0, "channel": 0},
        {"center": [0.7, 0.5, 0.4], "radius": 0.15, "amplitude": 0.5, "channel": 1}]}},
    {"pattern": {"type": "Shell", "center": [0.5, 0.5, 0.5], "inner_radius": 0.1, "outer_radius": 0.3,
                 "amplitude": 1.0, "channel": 0}},
    {"pattern": {"type": "Torus3D", "center": [0.5, 0.5, 0.5], "major_radius": 0.25, "minor_radius": 0.08,
                 "amplitude": 1.0, "channel": 1}},
    {"pattern": {"type": "GaussianBlob", "center": [0.5, 0.5], "radius": 0.2, "amplitude": 1.0, "channel": 0}},
    {"pattern": {"type": "Custom3D", "values": [[1, 2, 3, 0, 0.5], [15, 11, 9, 1, 0.25]]}},
]


@pytest.mark.parametrize("seed", SEEDS_2D)
def test_seed_generation_bit_exact_2d(seed):
    """Seed::generate (seed.rs:160-304) — engine host code vs oracle, bit for bit."""
    cfg = wl.config(48, 40, 2, [wl.kernel()])
    st = fl.SimulationState.from_seed(seed, cfg)
    assert np.array_equal(st.channels, O.seed_generate(seed, cfg))


@pytest.mark.parametrize("seed", SEEDS_3D)
def test_seed_generation_bit_exact_3d(seed):
    cfg = wl.config(16, 12, 2, [wl.kernel()], depth=10)
    st = fl.SimulationState.from_seed(seed, cfg)
    assert np.array_equal(st.channels, O.seed_generate(seed, cfg))


def test_state_total_mass_is_reference_f32_order():
    cfg, seed = wl.single_blob(64)
    st = fl.SimulationState.from_seed(seed, cfg)
    assert st.total_mass() == O.total_mass(st.channels.reshape(-1))


@pytest.mark.parametrize("bad", [
    {"width": 0}, {"channels": 0}, {"dt": 0.0}, {"dt": -0.1}, {"kernel_radius": 0},
    {"kernels": [wl.kernel(src=0, tgt=2)]}, {"kernels": [wl.kernel(src=5, tgt=0)]},
])
def test_invalid_config_rejected(bad):
    """config.rs:136-164 — rejected with INVALID_CONFIG before any device work."""
    cfg = dict(wl.config(32, 32, 1, [wl.kernel()]), **bad)
    with pytest.raises(fl.ConfigError):
        fl.SimulationState.from_seed(SEEDS_2D[0], cfg)


def test_malformed_json_rejected():
    out = np.zeros(4, np.float32)
    rc = nat.lib().flp_seed_generate(b"{not json", b"{}", out.ctypes.data, 4)
    assert rc == -1 and b"JSON" in nat.lib().flp_last_error()


def test_unknown_pattern_rejected():
    cfg = wl.config(8, 8, 1, [wl.kernel()])
    with pytest.raises(fl.ConfigError):
        fl.SimulationState.from_seed({"pattern": {"type": "Nope"}}, cfg)


def test_reference_example_files_parse():
    """The reference's example configs use the same schema (examples/*.json)."""
    glider = {"width": 128, "height": 128, "channels": 1, "dt": 0.2, "kernel_radius": 13,
              "kernels": [wl.kernel()], "flow": {"beta_a": 1.0, "n": 2.0, "distribution_size": 1.0},
              "embedding": {"enabled": False, "mixing_temperature": 1.0, "linear_mixing": False}}
    st = fl.SimulationState.from_seed(json.dumps(SEEDS_2D[0]), json.dumps(glider))
    assert st.channels.shape == (1, 128 * 128)


def test_no_cpu_fallback_without_device():
    """Creating a propagator needs the CUDA device; without one it raises."""
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("device present")
    cfg, _ = wl.single_blob(32)
    with pytest.raises(fl.FlpError):
        fl.CudaPropagator(cfg)


def test_batch_layout_match_rules():
    """BatchedPropagator.layout_matches: reconfigure keeps sides, channels and
    the kernels' (source, target) pairs; every other parameter may change."""
    from autoverse_b200 import workloads as wl
    from autoverse_b200.batch import BatchedPropagator
    from autoverse_b200.propagator import SimulationConfig
    worlds = wl.batched_worlds(4, sides=(64, 96), seed=1)
    b = BatchedPropagator.__new__(BatchedPropagator)  # layout logic only: no device batch
    b.configs = [SimulationConfig.load(c) for c, _ in worlds]
    nxt = wl.mutated_worlds(worlds, 2)
    assert b.layout_matches([c for c, _ in nxt])
    assert not b.layout_matches([c for c, _ in nxt][:3])
    other = [dict(c) for c, _ in nxt]
    other[0] = dict(other[0], height=other[0]["height"] * 2)
    assert not b.layout_matches(other)
    two = next(i for i, (c, _) in enumerate(nxt) if c["channels"] == 2)  # kernels (0,0), (0,1), (1,0), (1,1)
    swapped = [SimulationConfig.load(c) for c, _ in nxt]
    ks = swapped[two]["kernels"]
    ks[0], ks[1] = ks[1], ks[0]
    assert not b.layout_matches(swapped)


def test_twin64_rejects_before_device_work():
    """flp_twin64_step checks its arguments and the config on the host before
    it touches the device: a null buffer, an invalid config and a 3D world
    (the twin covers 2D steps) are refused with their codes."""
    lib = nat.lib()
    cfg = wl.config(16, 16, 1, [wl.kernel()])
    a = np.zeros(16 * 16, np.float64)
    out = np.zeros_like(a)
    rc = lib.flp_twin64_step(json.dumps(cfg).encode(), None, None, out.ctypes.data)
    assert rc == -2
    bad = dict(cfg, dt=0.0)
    rc = lib.flp_twin64_step(json.dumps(bad).encode(), a.ctypes.data, None, out.ctypes.data)
    assert rc == -1 and b"Time step" in lib.flp_last_error()
    cube = dict(cfg, depth=32, width=32, height=32)
    rc = lib.flp_twin64_step(json.dumps(cube).encode(), a.ctypes.data, None, out.ctypes.data)
    assert rc == -7 and b"2D" in lib.flp_last_error()
