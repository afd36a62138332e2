"""3D worlds on the GPU against the oracle's restatement of CpuPropagator3D
(src/compute/propagator3d.rs:119-308): the 3D transport stage bit-exact given
the same affinity; full steps within 1e-5 (1 step) and 1e-4 (10 steps)."""
import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import workloads as wl
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def sphere_case(W=32, H=32, D=32, R=5, C=1, seed=0, steps_in=2, **flow):
    cfg, sd = wl.sphere3d(W, R=R, radius=0.2)
    cfg.update(width=W, height=H, depth=D)
    if C == 2:
        cfg["channels"] = 2
        cfg["kernels"] = [wl.kernel(0, 0), wl.kernel(1, 1, mu=0.2, sigma=0.02), wl.kernel(0, 1, weight=0.5)]
        sd = {"pattern": {"type": "MultiSphere", "spheres": [
            {"center": [0.4, 0.5, 0.5], "radius": 0.2, "amplitude": 1.0, "channel": 0},
            {"center": [0.6, 0.5, 0.45], "radius": 0.15, "amplitude": 0.8, "channel": 1}]}}
    cfg["flow"].update(flow)
    st = O.seed_generate(sd, cfg)
    if steps_in:
        st = O.OraclePropagator(cfg).run(st, steps_in)
    return cfg, st


def noise_case(W=32, H=48, D=32, seed=3):
    """Mass in every cell (0.05 + U(0, 0.1)): every destination's window and
    every wrapped window order across all six faces carries nonzero terms."""
    cfg, _ = sphere_case(W, H, D, R=4, steps_in=0)
    st = (0.05 + 0.1 * np.random.default_rng(seed).random((1, W * H * D))).astype(np.float32)
    return cfg, st


def corner_case():
    """A sphere centred on a corner of the torus, spread over all eight octants."""
    cfg, _ = sphere_case(steps_in=0)
    sd = {"pattern": {"type": "GaussianSphere", "center": [0.02, 0.97, 0.01], "radius": 0.2, "amplitude": 1.0,
                      "channel": 0}}
    st = O.OraclePropagator(cfg).run(O.seed_generate(sd, cfg), 2)
    return cfg, st


def many_channels_case(C=8, seed=5):
    """C channels (each with its own kernel and one cross kernel from the
    previous channel) on a 32^3 torus filled with low-amplitude noise: the
    flow pass stages 2C+1 blocks (about 136 KB of shared memory at C=8 with
    four planes per CTA; at C=16 it falls back to two planes, 181 KB)."""
    rng = np.random.default_rng(seed)
    ks = [wl.kernel(c, c, mu=float(rng.uniform(0.1, 0.2)), sigma=0.02) for c in range(C)]
    ks += [wl.kernel(c - 1, c, weight=0.5) for c in range(1, C)]
    cfg = wl.config(32, 32, C, ks, kernel_radius=4, depth=32)
    st = (0.02 + 0.05 * rng.random((C, 32 * 32 * 32))).astype(np.float32)
    return cfg, st


CASES = {
    "cube32": lambda: sphere_case(),
    "box48x32x64_2ch": lambda: sphere_case(48, 32, 64, R=4, C=2, seed=1),
    "cube32_s05": lambda: sphere_case(distribution_size=0.5),
    "cube32_s075_n3": lambda: sphere_case(distribution_size=0.75, n=3.0),
    "box32x48x32_noise": noise_case,
    "cube32_corner": corner_case,
    "cube32_8ch_noise": many_channels_case,
    "cube32_16ch_noise": lambda: many_channels_case(C=16, seed=6),  # two planes per flow CTA (above 13 channels)
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_transport3d_bit_exact(name):
    cfg, st = CASES[name]()
    orc = O.OraclePropagator(cfg)
    aff = orc.affinity(st)
    exp = orc.transport(st, aff)
    with fl.CudaPropagator(cfg) as p:
        got = p.debug_transport(st, aff)
    assert np.array_equal(got, exp), f"max diff {np.abs(got - exp).max()}"


@pytest.mark.parametrize("name", ["cube32", "box48x32x64_2ch"])
def test_step3d_parity_1_and_10(name):
    cfg, st = CASES[name]()
    orc = O.OraclePropagator(cfg)
    with fl.CudaPropagator(cfg) as p:
        state = fl.SimulationState(st, cfg["width"], cfg["height"], cfg["depth"])
        p.step(state)
        e1 = orc.run(st, 1)
        assert np.abs(state.channels - e1).max() <= 1e-5
        p.run(state, 9)
        e10 = orc.run(e1, 9)
        assert np.abs(state.channels - e10).max() <= 1e-4


def test_affinity3d_close_to_fp64():
    cfg, st = sphere_case(64, 64, 64, R=10)
    exp32 = O.OraclePropagator(cfg).affinity(st)
    exp64 = O.OraclePropagator(cfg, f64=True).affinity(st.astype(np.float64))
    with fl.CudaPropagator(cfg) as p:
        p.write_state(st)
        got = p.debug_affinity()
    err_orc = np.abs(exp32 - exp64).max()
    err_gpu = np.abs(got - exp64).max()
    assert err_gpu <= 4.0 * err_orc + 2e-6, (err_gpu, err_orc)


def test_mass3d_conservation():
    cfg, st = sphere_case(steps_in=0)
    with fl.CudaPropagator(cfg) as p:
        p.write_state(st)
        m0 = p.total_mass()
        p.run_device(50)
        p.synchronize()
        assert abs(p.total_mass() - m0) / m0 < 1e-4


def test_3d_channel_limit_is_refused():
    """A 3D world whose stencil staging does not fit one CTA's shared memory
    is refused at creation with UNSUPPORTED, not at its first launch."""
    cfg, _ = sphere_case(steps_in=0)
    cfg["channels"] = 21
    with pytest.raises(fl._native.FlpError, match="at most 20 channels"):
        fl.CudaPropagator(cfg)


def test_3d_depth_outside_the_transform_sizes_is_refused():
    """3D depths are the z-transform sizes 32, 48, 64, 96, 128, 192 and 256,
    all multiples of 16, so the flow pass's plane blocks (4 or 2 planes) always
    divide the depth; any other depth (54 here) is refused at creation."""
    cfg, _ = sphere_case(32, 32, 32, steps_in=0)
    cfg["depth"] = 54
    with pytest.raises(fl._native.FlpError, match="D in"):
        fl.CudaPropagator(cfg)
