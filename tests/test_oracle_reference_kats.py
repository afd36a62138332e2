"""The reference crate's own hot-path unit tests, run against the CPU oracle.

Each test restates one `#[test]` of the reference (file:line given) with its
inputs and thresholds, and runs it on the f32 oracle (and, where the reference
test is about precision-independent behaviour, on the f64 twin as well).  These
known-answer tests are what pins the oracle: the reference ships no golden
arrays and cannot be built here (no Rust toolchain).
"""
import math

import numpy as np
import pytest

from autoverse_b200 import workloads as wl
from oracle import oracle as O

RING = {"amplitude": 1.0, "distance": 0.5, "width": 0.15}
KCFG = {"radius": 1.0, "rings": [RING], "weight": 1.0, "mu": 0.15, "sigma": 0.015,
        "source_channel": 0, "target_channel": 0}


def prop_config(W=64, H=64, C=1, R=10, kernels=None):
    """propagator.rs:481-509 test_config()."""
    return {"width": W, "height": H, "depth": 1, "channels": C, "dt": 0.2, "kernel_radius": R,
            "kernels": kernels or [dict(KCFG)],
            "flow": {"beta_a": 1.0, "n": 2.0, "distribution_size": 1.0}}


# --------------------------------------------------------------------- kernel.rs

@pytest.mark.parametrize("f64", [False, True])
def test_kernel_normalization(f64):
    """kernel.rs:143-164"""
    k = O.kernel_build(KCFG, 10, f64=f64)
    assert abs(np.sum(k, dtype=k.dtype) - 1.0) < 1e-5


def test_kernel_symmetry():
    """kernel.rs:166-184"""
    k = O.kernel_build(KCFG, 10)
    c = k.shape[0] // 2
    for d in range(1, c):
        v1, v2, v3, v4 = k[c, c + d], k[c, c - d], k[c + d, c], k[c - d, c]
        assert abs(v1 - v2) < 1e-6 and abs(v1 - v3) < 1e-6 and abs(v1 - v4) < 1e-6


def test_kernel3d_normalization_symmetry_padding():
    """kernel3d.rs:159-246"""
    k = O.kernel_build(KCFG, 8, dims=3)
    assert abs(np.sum(k, dtype=np.float32) - 1.0) < 1e-5
    c = k.shape[0] // 2
    for d in range(1, c):
        v = k[c, c, c + d]
        for w in (k[c, c, c - d], k[c, c + d, c], k[c, c - d, c], k[c + d, c, c], k[c - d, c, c]):
            assert abs(v - w) < 1e-6
    k4 = O.kernel_build(KCFG, 4, dims=3)
    padded = O.kernel_pad(k4, 16, 16, 16)
    assert abs(np.sum(k4, dtype=np.float32) - np.sum(padded, dtype=np.float32)) < 1e-5


def test_kernel_pad_overwrite_when_wider_than_grid():
    """kernel.rs:98-117: taps that wrap onto the same cell overwrite (later wins)."""
    k = O.kernel_build(KCFG, 6)  # 13x13 onto 8x8
    p = O.kernel_pad(k, 8, 8)
    exp = np.zeros((8, 8), np.float32)
    for ky in range(13):
        for kx in range(13):
            exp[(ky - 6 + 8) % 8, (kx - 6 + 8) % 8] = k[ky, kx]
    assert np.array_equal(p, exp)


# --------------------------------------------------------------------- growth.rs

def test_growth_known_answers():
    """growth.rs:66-179"""
    assert abs(O.growth(0.15, 0.15, 0.015) - 1.0) < 1e-6
    assert abs(O.growth(1.0, 0.15, 0.015) + 1.0) < 0.01
    assert abs(O.growth(0.4, 0.5, 0.1) - O.growth(0.6, 0.5, 0.1)) < 1e-6
    grid = (np.arange(100) * np.float32(0.01)).astype(np.float32)
    for u in grid:
        g = O.growth(float(u), 0.15, 0.015)
        assert -1 - 1e-6 <= g <= 1 + 1e-6
    conv = np.array([0.1, 0.15, 0.2, 0.3], np.float32)
    t = O.growth_accumulate(conv, np.ones(4, np.float32), 0.5, 0.15, 0.015)
    for i in range(4):
        assert abs(t[i] - (1.0 + 0.5 * O.growth(float(conv[i]), 0.15, 0.015))) < 1e-6
    for i in range(1000):
        u = i * 0.01 - 5.0
        g = O.growth(u, 0.5, 0.1)
        assert -1 - 1e-6 <= g <= 1 + 1e-6
    assert O.growth(0.6, 0.5, 0.2) > O.growth(0.6, 0.5, 0.05)


# ------------------------------------------------------------------- gradient.rs

def test_sobel_uniform_and_ramps():
    """gradient.rs:114-158, 227-255"""
    gx, gy = O.sobel2d(np.ones((16, 16), np.float32))
    assert np.abs(gx).max() < 1e-6 and np.abs(gy).max() < 1e-6
    ramp = np.tile(np.arange(16, dtype=np.float32), (16, 1))
    gx, _ = O.sobel2d(ramp)
    assert (gx[1:-1, 1:-1] > 0).all()
    _, gy = O.sobel2d(ramp.T.copy())
    assert (gy[1:-1, :] > 0).all()


def test_sobel_matches_definition():
    """gradient.rs:160-187 (the looped Sobel and the fast one agree to 1e-6)."""
    W = H = 32
    g = (((np.arange(W * H) * 7) % 100) / np.float32(100.0)).astype(np.float32).reshape(H, W)
    gx, gy = O.sobel2d(g)
    sx = np.array([[-1, 0, 1], [-2, 0, 2], [-1, 0, 1]], np.float64)
    sy = sx.T
    ex = np.zeros((H, W))
    ey = np.zeros((H, W))
    for ky in range(3):
        for kx in range(3):
            v = np.roll(np.roll(g.astype(np.float64), -(ky - 1), 0), -(kx - 1), 1)
            ex += sx[ky, kx] * v
            ey += sy[ky, kx] * v
    assert np.abs(gx - ex * 0.125).max() < 1e-6
    assert np.abs(gy - ey * 0.125).max() < 1e-6


def test_sobel_periodic_and_diagonal():
    """gradient.rs:257-339"""
    W = H = 16
    x = np.arange(W, dtype=np.float32)
    phase = (np.float32(2.0 * math.pi) * x / np.float32(W)).astype(np.float32)
    g = np.tile(np.sin(phase), (H, 1)).astype(np.float32)
    gx, gy = O.sobel2d(g)
    assert np.abs(gy).max() < 1e-5
    cs = np.cos(phase)
    for xi in range(W):
        if abs(cs[xi]) > 0.3:
            assert (gx[:, xi] * cs[xi] > 0).all()
    yy, xx = np.meshgrid(np.arange(H), np.arange(W), indexing="ij")
    d = np.sin(2 * np.pi * xx / W + 2 * np.pi * yy / H).astype(np.float32)
    gx, gy = O.sobel2d(d)
    assert abs(np.abs(gx).sum() / np.abs(gy).sum() - 1.0) < 0.2


def test_sobel3d_known_answers():
    """gradient3d.rs:164-315"""
    gx, gy, gz = O.sobel3d(np.ones((8, 8, 8), np.float32))
    assert max(np.abs(gx).max(), np.abs(gy).max(), np.abs(gz).max()) < 1e-6
    s = 8
    ph = (2 * np.pi * np.arange(s) / s).astype(np.float32)
    g = np.broadcast_to(np.sin(ph), (s, s, s)).astype(np.float32).copy()
    gx, gy, gz = O.sobel3d(g)
    assert np.abs(gy).max() < 1e-4 and np.abs(gz).max() < 1e-4
    assert (gx[:, :, 1] > 0).all()
    s = 16
    z, y, x = np.meshgrid(*(np.arange(s, dtype=np.float32),) * 3, indexing="ij")
    c = s / 2
    g = np.exp(-((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2) / 20.0).astype(np.float32)
    gx, gy, gz = O.sobel3d(g)
    m = s // 2
    assert abs(gx[m, m, m]) < 0.1 and abs(gy[m, m, m]) < 0.1 and abs(gz[m, m, m]) < 0.1
    assert gx[m, m, m + 2] < 0.0


# ----------------------------------------------------------------------- flow.rs

def test_alpha_known_answers():
    """flow.rs:158-268"""
    beta, n = 2.0, 4.0  # FlowConfig::default()
    assert O.alpha(0.0, beta, n) == 0.0
    assert O.alpha(beta, beta, n) == 1.0
    assert O.alpha(2 * beta, beta, n) == 1.0
    vals = [O.alpha(m, 1.0, 2.0) for m in (0.0, 0.25, 0.5, 0.75, 1.0)]
    assert all(a < b for a, b in zip(vals, vals[1:]))
    assert abs(vals[2] - 0.25) < 1e-6
    assert abs(O.alpha(0.5, 1.0, 1.0) - 0.5) < 1e-6
    assert O.alpha(0.5, 1.0, 4.0) < O.alpha(0.5, 1.0, 2.0)
    assert abs(O.alpha(0.5, 1.0, 2.5) - 0.5 ** 2.5) < 1e-6


def test_flow_limits_and_stats():
    """flow.rs:175-215, 349-379"""
    gu = np.array([[1, 2, 3], [0.5, 1, 1.5]], np.float32)
    ga = np.array([[-1, -2, -3], [-0.5, -1, -1.5]], np.float32)
    f = O.flow_field(gu, ga, np.zeros(3, np.float32), 2.0, 4.0)
    assert np.abs(f - gu).max() < 1e-6
    f = O.flow_field(gu, ga, np.full(3, 20.0, np.float32), 2.0, 4.0)
    assert np.abs(f + ga).max() < 1e-6
    mean_alpha = np.mean([O.alpha(m, 1.0, 2.0) for m in (0.0, 0.5, 1.0)])
    assert abs(mean_alpha - (0 + 0.25 + 1) / 3) < 1e-5


# -------------------------------------------------------------- reintegration.rs

def test_wrap_coord_table():
    """reintegration.rs:293-301"""
    for c, e in [(0, 0), (5, 5), (10, 0), (-1, 9), (-10, 0), (15, 5)]:
        assert O.wrap_coord(c, 10) == e


def _flow(W, H, fx, fy):
    return np.full((H, W), fx, np.float32), np.full((H, W), fy, np.float32)


def test_reintegration_mass_conservation_cases():
    """reintegration.rs:234-470"""
    W = H = 16
    cur = np.zeros((H, W), np.float32)
    cur[8, 8], cur[7, 8] = 1.0, 0.5
    n = O.advect2d(cur, *_flow(W, H, 0, 0), 0.2, 1.0)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-5

    cur = np.zeros((32, 32), np.float32)
    cur[10:20, 10:20] = 1.0
    n = O.advect2d(cur, *_flow(32, 32, 5, 2), 0.2, 1.0)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-4

    cur = np.zeros((H, W), np.float32)
    cur[8, 14] = 1.0
    n = O.advect2d(cur, *_flow(W, H, 5, 0), 0.5, 1.0)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-5
    assert n[8, 0:3].sum() > 0.1 and n[8, 14] < 1.0

    cur = np.zeros((H, W), np.float32)
    cur[15, 15] = 1.0
    n = O.advect2d(cur, *_flow(W, H, 8, 8), 0.5, 1.0)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-5

    for c, (y, x, m) in enumerate([(8, 8, 1.0), (4, 4, 2.0)]):
        cur = np.zeros((H, W), np.float32)
        cur[y, x] = m
        n = O.advect2d(cur, *_flow(W, H, 2, 1), 0.2, 1.0)
        assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-5

    cur = np.zeros((H, W), np.float32)
    cur[8, 8] = 1.0
    n = O.advect2d(cur, *_flow(W, H, 100, 50), 0.2, 1.0)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-5

    n = O.advect2d(cur, *_flow(W, H, 1, 0), 0.2, 0.01)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-4


def test_reintegration3d_mass_conservation_cases():
    """reintegration3d.rs:240-456"""
    s = 8
    cur = np.zeros((s, s, s), np.float32)
    c = s // 2
    cur[c, c, c], cur[c, c, c - 1], cur[c, c + 1, c] = 1.0, 0.5, 0.3
    z = np.zeros_like(cur)
    n = O.advect3d(cur, z, z, z, 0.2, 1.0)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-5

    cur = np.zeros((16,) * 3, np.float32)
    cur[4:8, 4:8, 4:8] = 1.0
    f = [np.full_like(cur, v) for v in (3.0, 2.0, 1.0)]
    n = O.advect3d(cur, *f, 0.2, 1.0)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-4

    cur = np.zeros((s,) * 3, np.float32)
    cur[4, 4, s - 1] = 1.0
    f = [np.full_like(cur, v) for v in (5.0, 0.0, 0.0)]
    n = O.advect3d(cur, *f, 0.5, 1.0)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-5
    assert n[4, 4, 0:3].sum() > 0.1

    cur = np.zeros((s,) * 3, np.float32)
    cur[s - 1, s - 1, s - 1] = 1.0
    f = [np.full_like(cur, 4.0)] * 3
    n = O.advect3d(cur, *f, 0.5, 1.0)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-5

    cur = np.zeros((s,) * 3, np.float32)
    cur[c, c, c] = 1.0
    f = [np.full_like(cur, v) for v in (1.0, 0.0, 0.0)]
    n = O.advect3d(cur, *f, 0.2, 0.01)
    assert abs(O.total_mass(cur) - O.total_mass(n)) < 1e-4


# ------------------------------------------------------------------------ fft.rs

def test_fft_roundtrip_and_sizes():
    """fft.rs:492-509, 660-683"""
    for W, H in [(16, 16), (8, 8), (32, 32), (16, 32), (32, 16)]:
        x = (np.arange(W * H) % 10).astype(np.float32).reshape(H, W)
        r = O.fft_inverse(O.fft_forward(x))
        assert np.abs(r - x).max() < 1e-4


def test_fft_convolution_known_answers():
    """fft.rs:511-658"""
    W = H = 16
    x = np.zeros((H, W), np.float32)
    x.flat[W * H // 2 + W // 2] = 1.0
    k = np.zeros((H, W), np.float32)
    k[0, 0] = 1.0
    assert np.abs(O.fft_convolve(x, k) - x).max() < 1e-4
    x = np.zeros((H, W), np.float32)
    x[5, 5] = 1.0
    k = np.zeros((H, W), np.float32)
    k[2, 3] = 1.0
    r = O.fft_convolve(x, k)
    assert abs(r[7, 8] - 1.0) < 1e-4 and abs(r.sum() - 1.0) < 1e-4
    x = np.zeros((H, W), np.float32)
    x[8, 8] = 1.0
    k = np.zeros((H, W), np.float32)
    for ky in range(3):
        for kx in range(3):
            wy = 0 if ky == 0 else H - (3 - ky)
            wx = 0 if kx == 0 else W - (3 - kx)
            k[wy, wx] = np.float32(1.0 / 9.0)
    r = O.fft_convolve(x, k)
    assert abs(r.sum() - 1.0) < 1e-4 and 0.05 < r[8, 8] < 0.5
    a = (((np.arange(W * H) * 17) % 100) / np.float32(100.0)).astype(np.float32).reshape(H, W)
    b = (((np.arange(W * H) * 31 + 7) % 100) / np.float32(100.0)).astype(np.float32).reshape(H, W)
    assert np.abs(O.fft_convolve(a, b) - O.fft_convolve(b, a)).max() < 1e-4


def test_fft_vs_direct_convolution():
    """fft.rs:718-787: max |FFT - direct| < 1e-4 at 64x64, R=7."""
    W = H = 64
    k = O.kernel_build(KCFG, 7)
    yy, xx = np.meshgrid(np.arange(H, dtype=np.float32), np.arange(W, dtype=np.float32), indexing="ij")
    x = np.exp(-((xx - 32) ** 2 + (yy - 32) ** 2) / np.float32(50.0)).astype(np.float32)
    fr = O.fft_convolve(x, O.kernel_pad(k, W, H))
    dr = O.direct_convolve2d(x, k, 7)
    assert np.abs(fr - dr).max() < 1e-4


def test_fft3d_known_answers():
    """fft3d.rs:578-710"""
    s = 8
    x = (np.arange(s ** 3) % 10).astype(np.float32).reshape(s, s, s)
    assert np.abs(O.fft_inverse(O.fft_forward(x)) - x).max() < 1e-4
    x = np.zeros((s,) * 3, np.float32)
    x[4, 4, 4] = 1.0
    k = np.zeros_like(x)
    k[0, 0, 0] = 1.0
    assert np.abs(O.fft_convolve(x, k) - x).max() < 1e-4
    z, y, xx = np.meshgrid(*(np.arange(s, dtype=np.float32),) * 3, indexing="ij")
    g = np.exp(-((xx - 4) ** 2 + (y - 4) ** 2 + (z - 4) ** 2) / 8.0).astype(np.float32)
    k = np.zeros_like(g)
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                wz = 0 if kz == 0 else s - (3 - kz)
                wy = 0 if ky == 0 else s - (3 - ky)
                wx = 0 if kx == 0 else s - (3 - kx)
                k[wz, wy, wx] = np.float32(1.0 / 27.0)
    assert abs(np.sum(g, dtype=np.float32) - np.sum(O.fft_convolve(g, k), dtype=np.float32)) < 1e-3
    k4 = O.kernel_build(KCFG, 4, dims=3)
    x = np.zeros((16,) * 3, np.float32)
    x[8, 8, 8] = 1.0
    out = O.fft_convolve(x, O.kernel_pad(k4, 16, 16, 16))
    assert out.sum() > 0 and abs(out.sum() - 1.0) < 0.01


# ----------------------------------------------------------------- propagator.rs

def test_propagator_mass_conservation_10_and_100_steps():
    """propagator.rs:517-548 (<1% over 10 steps) and 561-592 (<0.1% over 100)."""
    cfg = prop_config()
    seed = {"pattern": {"type": "GaussianBlob", "center": [0.5, 0.5], "radius": 0.15, "amplitude": 1.0,
                        "channel": 0}}
    st = O.seed_generate(seed, cfg)
    m0 = O.total_mass(st)
    p = O.OraclePropagator(cfg)
    s10 = p.run(st, 10)
    assert abs(O.total_mass(s10) - m0) / m0 < 0.01
    s100 = p.run(s10, 90)
    assert abs(O.total_mass(s100) - m0) / m0 < 0.001


def test_state_from_seed_default():
    """propagator.rs:550-559"""
    cfg = prop_config()
    seed = {"pattern": {"type": "GaussianBlob", "center": [0.5, 0.5], "radius": 0.1, "amplitude": 1.0,
                        "channel": 0}}
    st = O.seed_generate(seed, cfg)
    assert st.shape == (1, 64 * 64) and O.total_mass(st) > 0


def test_propagator_multichannel_mass():
    """propagator.rs:594-676"""
    k0 = dict(KCFG)
    k1 = dict(KCFG, source_channel=1, target_channel=1)
    cfg = prop_config(C=2, kernels=[k0, k1])
    seed = {"pattern": {"type": "MultiBlob", "blobs": [
        {"center": [0.3, 0.5], "radius": 0.1, "amplitude": 1.0, "channel": 0},
        {"center": [0.7, 0.5], "radius": 0.1, "amplitude": 2.0, "channel": 1}]}}
    st = O.seed_generate(seed, cfg)
    out = O.OraclePropagator(cfg).run(st, 20)
    for c in range(2):
        m0 = np.sum(st[c], dtype=np.float32)
        m1 = np.sum(out[c], dtype=np.float32)
        assert abs(m1 - m0) / m0 < 0.01


def test_propagator3d_mass_and_seed():
    """propagator3d.rs:369-458"""
    cfg = {"width": 16, "height": 16, "depth": 16, "channels": 1, "dt": 0.2, "kernel_radius": 4,
           "kernels": [dict(KCFG)], "flow": {"beta_a": 1.0, "n": 2.0, "distribution_size": 1.0}}
    seed = {"pattern": {"type": "GaussianSphere", "center": [0.5, 0.5, 0.5], "radius": 0.2, "amplitude": 1.0,
                        "channel": 0}}
    st = O.seed_generate(seed, cfg)
    assert st.shape == (1, 16 ** 3) and O.total_mass(st) > 0
    out = O.OraclePropagator(cfg).run(st, 5)
    m0 = O.total_mass(st)
    assert abs(O.total_mass(out) - m0) / m0 < 0.02


def test_config_validation():
    """config.rs:136-164"""
    base = prop_config()
    for field, val in [("width", 0), ("channels", 0), ("dt", 0.0), ("kernel_radius", 0)]:
        with pytest.raises(ValueError):
            O.validate_config(dict(base, **{field: val}))
    with pytest.raises(ValueError):
        O.validate_config(dict(base, kernels=[dict(KCFG, target_channel=3)]))


def test_mass_drift_comes_from_rounding_and_the_skip():
    """Where the reference's mass drift comes from, on a 96x96 blob over 1000
    steps: the FP64 twin without the |m| < 1e-10 skip of the reintegration
    (reintegration.rs:74-76) conserves mass to FP64 round-off; with the skip
    it loses a little (the blob's far tail); the f32 reference loses more,
    from the rounding of its f32 overlap areas and sums."""
    cfg, sd = wl.single_blob(96, R=13, blob_radius=0.1)
    st = O.seed_generate(sd, cfg)
    m0 = st.astype(np.float64).sum()
    drift = {}
    for name, kw in (("noskip", dict(f64=True, mass_skip=False)), ("f64", dict(f64=True)), ("f32", {})):
        a = O.OraclePropagator(cfg, **kw).run(st.astype(np.float64 if kw else np.float32), 1000)
        drift[name] = abs(a.astype(np.float64).sum() - m0) / m0
    assert drift["noskip"] < 1e-13
    assert drift["f64"] > 1e3 * drift["noskip"]
    assert drift["f32"] > drift["f64"]
