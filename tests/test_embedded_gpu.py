"""Parameter-embedded worlds on the GPU (flp_emb_*) against the oracle's
restatement of EmbeddedPropagator::step (src/compute/embedded_propagator.rs:
222-339).  Growth and softmax weights go through expf (and powf for
non-integer n), whose last bit may differ from the host's libm, so state and
parameters are compared within 1e-5 after one step and 1e-4 after ten (the
same bar as the plain engine); the direct convolution sum, the overlap
areas and the mixing arithmetic follow the reference's operation order.
Kernels of radius >= 8 on FFT grids (the R = 9, 10 and 12 cases) take the FFT
convolution, whose sums differ from the direct ones by f32 rounding."""
import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import workloads as wl
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def species_params(cfg, rng):
    """Two species (left/right halves) with distinct CellParams per channel."""
    W, H, C = cfg["width"], cfg["height"], cfg["channels"]
    prm = np.empty((C, H, W, 5), np.float32)
    a = np.float32([0.14, 0.016, 1.0, 1.0, 2.0])
    b = np.float32([0.2, 0.03, 1.4, 0.8, 2.5])   # non-integer n: the powf path
    prm[:, :, : W // 2] = a
    prm[:, :, W // 2:] = b
    prm += rng.uniform(-1e-3, 1e-3, prm.shape).astype(np.float32) * np.float32([1, 0.1, 1, 1, 0])
    return prm.reshape(C, H * W, 5)


def emb_case(W=64, H=48, C=2, R=7, enabled=True, linear=False, temperature=1.0, seed=1, dt=0.2, s=1.0):
    rng = np.random.default_rng(seed)
    ks = [wl.kernel(src=i, tgt=j, rings=wl.random_rings(rng), mu=0.15, sigma=0.015)
          for i in range(C) for j in range(C)]
    cfg = wl.config(W, H, C, ks, kernel_radius=R, dt=dt, s=s)
    cfg["embedding"] = {"enabled": enabled, "mixing_temperature": temperature, "linear_mixing": linear}
    st = np.zeros((C, H, W), np.float32)
    for c in range(C):
        for _ in range(4):
            x, y = rng.integers(0, W - 12), rng.integers(0, H - 12)
            st[c, y:y + 12, x:x + 12] = rng.random((12, 12), dtype=np.float32)
    return cfg, st.reshape(C, -1), species_params(cfg, rng)


CASES = {
    "softmax": lambda: emb_case(),
    "linear": lambda: emb_case(seed=2, linear=True),
    "cold_softmax": lambda: emb_case(seed=3, temperature=0.05),
    "one_channel_square": lambda: emb_case(48, 48, C=1, R=9, seed=4),
    "disabled": lambda: emb_case(seed=5, enabled=False),
    "s075": lambda: emb_case(seed=6, s=0.75),
    # kernels of radius >= 8 on these grids take the FFT convolution
    "fft_two_channel": lambda: emb_case(64, 48, C=2, R=10, seed=13),
    "fft_linear_s075": lambda: emb_case(64, 64, C=1, R=12, seed=14, linear=True, s=0.75),
}


def gpu_run(cfg, st, prm, steps):
    with fl.EmbeddedPropagator(cfg) as p:
        p.write(fl.EmbeddedState(st, prm, cfg["width"], cfg["height"]))
        p.run_device(steps)
        p.synchronize()
        out = p.read()
    return out


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("steps,tol", [(1, 1e-5), (10, 1e-4)])
def test_embedded_parity(name, steps, tol):
    cfg, st, prm = CASES[name]()
    ref_st, ref_prm = O.OracleEmbedded(cfg).run(st, prm, steps)
    out = gpu_run(cfg, st, prm, steps)
    assert out.step == steps
    assert np.abs(out.channels - ref_st).max() <= tol
    assert np.abs(out.params - ref_prm).max() <= tol * 10  # fields up to ~3 in size
    if not cfg["embedding"]["enabled"]:
        assert np.array_equal(out.params, prm)


def test_embedded_parameters_travel_with_mass():
    """A blob of species B moving through species A carries B's mu along."""
    cfg, st, prm = emb_case(seed=7)
    out = gpu_run(cfg, st, prm, 20)
    ref_st, ref_prm = O.OracleEmbedded(cfg).run(st, prm, 20)
    assert not np.array_equal(out.params, prm)
    massive = ref_st > 1e-3
    assert np.abs(out.params[massive] - ref_prm[massive]).max() < 1e-3


def test_embedded_stale_parameters_follow_the_buffer_swap():
    """Cells that receive no mass keep the propagator's other buffer
    (CellParams::default after the first step), bit for bit."""
    cfg, st, prm = emb_case(32, 32, C=1, R=5, seed=8)
    st = np.zeros_like(st)
    st[0, 16 * 32 + 16] = 1.0
    ref_st, ref_prm = O.OracleEmbedded(cfg).run(st, prm, 1)
    out = gpu_run(cfg, st, prm, 1)
    empty = ref_st[0] == 0
    assert empty.sum() > 900
    assert np.array_equal(out.params[0][empty], ref_prm[0][empty])
    assert np.allclose(out.params[0][empty], O.CELL_DEFAULT)


def test_embedded_edge_crossing_mass_is_lost_like_the_reference():
    """The reference places a wrapped source's square at its wrapped index
    (param_advection.rs:117-140), so mass pushed across the torus edge is not
    delivered; the engine keeps that."""
    cfg, st, prm = emb_case(32, 32, C=1, R=5, seed=9)
    st = np.zeros_like(st)
    st[0, 10 * 32 + 31] = 0.5
    st[0, 20 * 32 + 0] = 0.5
    ref_st, _ = O.OracleEmbedded(cfg).run(st, prm, 3)
    out = gpu_run(cfg, st, prm, 3)
    assert np.abs(out.channels - ref_st).max() < 1e-6


def test_embedded_from_seed_defaults_and_run_graph():
    cfg, _, _ = emb_case(seed=10)
    seed = {"pattern": {"type": "GaussianBlob", "center": [0.5, 0.5], "radius": 0.2, "amplitude": 1.0,
                        "channel": 0}}
    st = fl.EmbeddedState.from_seed(seed, cfg)
    k0, f = cfg["kernels"][0], cfg["flow"]
    want = np.float32([k0["mu"], k0["sigma"], k0["weight"], f["beta_a"], f["n"]])
    assert np.array_equal(st.params[0, 0], want) and st.channels.sum() > 0
    with fl.EmbeddedPropagator(cfg) as p1, fl.EmbeddedPropagator(cfg) as p2:
        p1.write(st)
        p2.write(st)
        p1.run_device(37)  # two graph replays and 5 single steps
        for _ in range(37):
            p2.run_device(1)
        a, b = p1.read(), p2.read()
        assert np.array_equal(a.channels, b.channels) and np.array_equal(a.params, b.params)
        assert a.step == 37 and a.time == pytest.approx(float(np.float32(0.2)) * 37, rel=1e-5)
        m = p1.total_mass()
    assert abs(m - a.channels.sum(dtype=np.float64)) / m < 1e-9


def test_embedded_step_api_matches_device_run():
    cfg, st, prm = emb_case(seed=11)
    state = fl.EmbeddedState(st, prm, cfg["width"], cfg["height"])
    with fl.EmbeddedPropagator(cfg) as p:
        p.step(state)
        p.step(state)
    out = gpu_run(cfg, st, prm, 2)
    assert np.array_equal(state.channels, out.channels) and state.step == 2


def test_embedded_rejects_3d_and_incomplete_embedding():
    cfg, _, _ = emb_case(seed=12)
    bad = dict(cfg, depth=4)
    with pytest.raises(fl.FlpError):
        fl.EmbeddedPropagator(bad)
    partial = dict(cfg, embedding={"enabled": True})
    with pytest.raises(fl.ConfigError):
        fl.EmbeddedPropagator(partial)
