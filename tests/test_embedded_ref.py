"""The EmbeddedPropagator oracle (per-cell parameters advected with mass)
against the reference's own tests for that path: schema/embedding.rs:416-470,
compute/param_advection.rs:311-472, compute/direct_convolution.rs:341-420 and
compute/embedded_propagator.rs:374-544.  CPU only."""
import numpy as np
import pytest

from autoverse_b200 import workloads as wl
from oracle import oracle as O


def cp(mu, sigma, weight, beta_a, n):
    return [mu, sigma, weight, beta_a, n]


# -- CellParams mixing (embedding.rs:416-450) ------------------------------

def test_mix_softmax_single_source():
    p = cp(0.2, 0.02, 1.5, 1.0, 2.0)
    assert np.array_equal(O.mix_softmax([1.0], [p]), np.float32(p))


def test_mix_softmax_equal_masses():
    m = O.mix_softmax([1.0, 1.0], [cp(0.1, 0.01, 1.0, 1.0, 2.0), cp(0.2, 0.02, 2.0, 2.0, 4.0)], 1.0)
    assert abs(m[0] - 0.15) < 1e-5 and abs(m[1] - 0.015) < 1e-5


def test_mix_linear_proportional():
    m = O.mix_linear([3.0, 1.0], [cp(0.1, 0.01, 1.0, 1.0, 2.0), cp(0.3, 0.03, 3.0, 3.0, 6.0)])
    assert abs(m[0] - (0.75 * 0.1 + 0.25 * 0.3)) < 1e-5


def test_mix_softmax_low_temperature_takes_the_heaviest():
    m = O.mix_softmax([1.0, 0.2], [cp(0.1, 0.01, 1.0, 1.0, 2.0), cp(0.3, 0.03, 3.0, 3.0, 6.0)], 0.01)
    assert abs(m[0] - 0.1) < 1e-6


# -- parameter advection (param_advection.rs:311-472) -----------------------

def test_advect_no_flow():
    W = H = 16
    mass = np.zeros(W * H, np.float32)
    mass[8 * W + 8] = 1.0
    params = np.tile(np.float32(O.CELL_DEFAULT), (W * H, 1))
    params[8 * W + 8] = cp(0.25, 0.025, 2.0, 1.5, 3.0)
    z = np.zeros(W * H, np.float32)
    nm, npr = O.advect_params2d(mass, params, z, z, W, H, 0.2, 1.0)
    assert abs(nm.sum() - 1.0) < 0.01
    assert abs(npr[8 * W + 8][0] - 0.25) < 0.1


def test_advect_with_flow():
    W = H = 32
    mass = np.zeros(W * H, np.float32)
    mass[16 * W + 10] = 1.0
    params = np.tile(np.float32(O.CELL_DEFAULT), (W * H, 1))
    custom = cp(0.3, 0.03, 1.5, 1.0, 2.0)
    params[16 * W + 10] = custom
    fx = np.full(W * H, 5.0, np.float32)
    fy = np.zeros(W * H, np.float32)
    nm, npr = O.advect_params2d(mass, params, fx, fy, W, H, 0.2, 1.0)
    assert abs(nm.sum() - 1.0) < 0.01
    assert nm[16 * W + 11] > 0 or nm[16 * W + 12] > 0
    if nm[16 * W + 11] > 0.1:
        assert abs(npr[16 * W + 11][0] - custom[0]) < 0.2


def test_mixing_collision():
    W = H = 16
    mass = np.zeros(W * H, np.float32)
    mass[8 * W + 4] = 1.0
    mass[8 * W + 10] = 1.0
    params = np.tile(np.float32(O.CELL_DEFAULT), (W * H, 1))
    params[8 * W + 4] = cp(0.1, 0.01, 1.0, 1.0, 2.0)
    params[8 * W + 10] = cp(0.3, 0.03, 1.0, 1.0, 2.0)
    fx = np.zeros(W * H, np.float32)
    fx[8 * W + 4] = 15.0
    fx[8 * W + 10] = -15.0
    fy = np.zeros(W * H, np.float32)
    nm, npr = O.advect_params2d(mass, params, fx, fy, W, H, 0.2, 1.0, linear=True)
    assert abs(nm.sum() - 2.0) < 0.01
    i = int(np.argmax(nm))
    if nm[i] > 0.5:
        assert 0.1 < npr[i][0] < 0.3


def test_distribution_overlap():
    assert O.distribution_overlap(0.5, 0.5, 2.0, 0.0, 0.0) > 0.0
    assert abs(O.distribution_overlap(10.0, 10.0, 1.0, 0.0, 0.0)) < 1e-6
    p = O.distribution_overlap(0.0, 0.0, 1.0, 0.0, 0.0)
    assert 0.0 < p < 1.0


def test_advect_loses_mass_across_the_torus_edge():
    """The reference's gather places a wrapped source's square at its wrapped
    index, so mass pushed across an edge is not delivered (param_advection.rs:
    117-140); the oracle keeps that behaviour."""
    W = H = 16
    mass = np.zeros(W * H, np.float32)
    mass[8 * W + 15] = 1.0
    params = np.tile(np.float32(O.CELL_DEFAULT), (W * H, 1))
    fx = np.full(W * H, 2.5, np.float32)  # dest x = 15.5: the square reaches past x = 16
    fy = np.zeros(W * H, np.float32)
    nm, _ = O.advect_params2d(mass, params, fx, fy, W, H, 0.2, 1.0)
    assert 0.0 < nm.sum() < 0.9


def test_untouched_cells_keep_the_buffer():
    """Destinations without mass keep what the output buffer held."""
    W = H = 8
    mass = np.zeros(W * H, np.float32)
    params = np.tile(np.float32(O.CELL_DEFAULT), (W * H, 1))
    prev = np.tile(np.float32([0.4, 0.04, 4.0, 4.0, 4.0]), (W * H, 1))
    z = np.zeros(W * H, np.float32)
    _, npr = O.advect_params2d(mass, params, z, z, W, H, 0.2, 1.0, next_params=prev)
    assert np.array_equal(npr, prev)


# -- direct convolution with per-cell growth (direct_convolution.rs:341-420) --

def test_convolve_growth_embedded():
    W = H = 8
    kern = O.kernel_build(wl.kernel(), 5)
    params = np.tile(np.float32(O.CELL_DEFAULT), (W * H, 1))
    out = O.conv_growth_embedded(np.full(W * H, 0.15, np.float32), kern, params, W, H)
    assert (out > 0.5).all()


def test_convolve_growth_embedded_varying_params():
    W = H = 16
    kcfg = {"radius": 1.0, "rings": [{"amplitude": 1.0, "distance": 0.5, "width": 0.15}], "weight": 1.0,
            "mu": 0.15, "sigma": 0.015, "source_channel": 0, "target_channel": 0}
    kern = O.kernel_build(kcfg, 5)
    params = np.tile(np.float32(O.CELL_DEFAULT), (H, W, 1))
    params[:, : W // 2, 0] = 0.2
    params[:, W // 2:, 0] = 0.5
    out = O.conv_growth_embedded(np.full(W * H, 0.2, np.float32), kern, params, W, H).reshape(H, W)
    assert out[:, : W // 2].mean() > out[:, W // 2:].mean()


def test_conv_matches_plain_direct_sum():
    """The embedded convolution's sum is the plain direct correlation (same
    order; zero taps only add signed zeros), followed by the growth with each
    cell's own parameters."""
    rng = np.random.default_rng(3)
    W, H = 24, 20
    kern = O.kernel_build(wl.kernel(), 4)
    x = rng.random(W * H).astype(np.float32)
    conv = O.direct_convolve2d(x.reshape(H, W), kern, kern.shape[0] // 2).reshape(-1)
    params = np.tile(np.float32(O.CELL_DEFAULT), (W * H, 1))
    params[:, 0] = rng.uniform(0.1, 0.3, W * H)
    params[:, 1] = rng.uniform(0.01, 0.05, W * H)
    params[:, 2] = rng.uniform(0.5, 2.0, W * H)
    g = O.conv_growth_embedded(x, kern, params, W, H)
    d = conv.astype(np.float64) - params[:, 0]
    want = params[:, 2] * (2 * np.exp(-d * d / (2.0 * params[:, 1] ** 2)) - 1)
    assert np.allclose(g, want, rtol=1e-5, atol=2e-6)


# -- the propagator (embedded_propagator.rs:374-544) -------------------------

def emb_config(W=32, H=32, C=1, R=5, enabled=True, linear=False, temperature=1.0):
    cfg = wl.config(W, H, C, [wl.kernel(src=c, tgt=c) for c in range(C)], kernel_radius=R)
    cfg["embedding"] = {"enabled": enabled, "mixing_temperature": temperature, "linear_mixing": linear}
    return cfg


def blob_state(cfg, cx=0.5, cy=0.5, r=0.15):
    seed = {"pattern": {"type": "GaussianBlob", "center": [cx, cy], "radius": r, "amplitude": 1.0, "channel": 0}}
    return O.seed_generate(seed, cfg).reshape(cfg["channels"], -1)


def test_embedded_state_defaults():
    cfg = emb_config()
    st = blob_state(cfg)
    prm = O.default_params(cfg)
    assert prm.shape == (1, 32 * 32, 5) and st.sum() > 0
    assert np.allclose(prm[0, 0], [0.15, 0.015, 1.0, 1.0, 2.0])


@pytest.mark.parametrize("enabled", [True, False])
def test_mass_conservation_embedded(enabled):
    cfg = emb_config(enabled=enabled)
    st = blob_state(cfg)
    prop = O.OracleEmbedded(cfg)
    m0 = float(st.sum(dtype=np.float64))
    st1, _ = prop.run(st, O.default_params(cfg), 10)
    assert abs(float(st1.sum(dtype=np.float64)) - m0) / m0 < 0.05


def test_parameter_advection_runs():
    cfg = emb_config()
    st = blob_state(cfg, cx=0.25, r=0.1)
    prm = O.default_params(cfg)
    cx, cy = int(32 * 0.25), int(32 * 0.5)
    prm[0, cy * 32 + cx] = cp(0.3, 0.03, 2.0, 1.5, 3.0)
    st1, prm1 = O.OracleEmbedded(cfg).run(st, prm, 5)
    assert prm1[0, cy * 32 + cx][0] > 0.0
    assert not np.array_equal(prm1, prm)


def test_disabled_embedding_keeps_parameters():
    cfg = emb_config(enabled=False)
    st = blob_state(cfg)
    prm = O.default_params(cfg)
    prm[0, :100, 0] = 0.2
    st1, prm1 = O.OracleEmbedded(cfg).run(st, prm, 3)
    assert np.array_equal(prm1, prm)


def test_disabled_embedding_moves_mass_like_the_plain_scatter():
    """With embedding off the mass moves by advect_mass_into, the plain
    propagator's scatter; with uniform default parameters and one kernel whose
    growth parameters equal the cells', the embedded step then differs from
    CpuPropagator only through the convolution (direct vs FFT)."""
    cfg = emb_config(enabled=False)
    st = blob_state(cfg)
    prm = O.default_params(cfg)
    st1, _ = O.OracleEmbedded(cfg).run(st, prm, 1)
    ref = O.OraclePropagator({k: v for k, v in cfg.items() if k != "embedding"}).run(st, 1)
    assert np.abs(st1 - ref).max() < 1e-4


def test_buffer_swap_leaves_stale_parameters_where_no_mass_arrives():
    """The propagator swaps its parameter buffer with the state's
    (embedded_propagator.rs:335-336), so a cell that receives no mass keeps the
    parameters the buffer held two steps earlier (CellParams::default after the
    first step)."""
    cfg = emb_config(W=16, H=16)
    st = np.zeros((1, 256), np.float32)
    st[0, 8 * 16 + 8] = 1.0
    prm = np.tile(np.float32([0.3, 0.03, 1.0, 1.0, 2.0]), (1, 256, 1))
    prop = O.OracleEmbedded(cfg)
    st1, prm1 = prop.run(st, prm, 1)
    far = 0  # (0, 0) receives nothing
    assert np.allclose(prm1[0, far], O.CELL_DEFAULT)
    assert np.allclose(prop.next_params()[0, far], [0.3, 0.03, 1.0, 1.0, 2.0])
