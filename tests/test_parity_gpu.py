"""GPU parity of the CUDA engine against the CPU oracle (restatement of the
reference's CpuPropagator), called through the C ABI.

Tolerances (f32 state):
* transport stage (channel sum, Sobel, alpha, flow, reintegration): bit-exact
  given the same affinity field, whenever the gather radius leaves the
  reference's deposit order intact (2R+1 <= min side); otherwise 1e-6 relative;
* affinity U: the GPU FFT/direct convolutions and the oracle's FFT round
  differently; both are compared with the FP64 oracle and the GPU may not be
  worse than AFF_FACTOR x the f32 oracle's own error plus AFF_ABS;
* full step: max |A_gpu - A_oracle| <= 1e-5 after 1 step, <= 1e-4 after 10.
"""
import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import workloads as wl
from oracle import oracle as O

pytestmark = pytest.mark.gpu

AFF_FACTOR = 4.0
AFF_ABS = 2e-6
STEP1_TOL = 1e-5
STEP10_TOL = 1e-4


def blob_case(size=64, R=10, steps_in=5, height=None):
    cfg, seed = wl.single_blob(size, R=R, blob_radius=0.15, height=height)
    st = O.seed_generate(seed, cfg)
    if steps_in:
        st = O.OraclePropagator(cfg).run(st, steps_in)
    return cfg, st


def species_case(W=96, H=64, C=3, R=9, seed=1, patches=6, patch=16, **flow):
    cfg, st = wl.multispecies(W, channels=C, R=R, patches=patches, patch=patch, seed=seed, height=H)
    cfg["flow"].update(flow)
    return cfg, st


def noise_case(W, H, C=2, seed=11):
    """Mass in every cell (0.05 + U(0, 0.1)): every gather tile's edge threads,
    both torus edges and every wrapped window order carry nonzero terms.
    Widths divisible by 4 take the one-sided edge column ranges, others the
    generic wrap passes."""
    cfg, _ = species_case(W=W, H=H, C=C, seed=seed)
    st = (0.05 + 0.1 * np.random.default_rng(seed).random((C, W * H))).astype(np.float32)
    return cfg, st


TRANSPORT_CASES = {
    "noise64x48": lambda: noise_case(64, 48),
    "noise68x40": lambda: noise_case(68, 40, seed=12),
    "noise70x36": lambda: noise_case(70, 36, seed=13),
    "noise36x36": lambda: noise_case(36, 36, seed=14),
    "noise100x52_1ch": lambda: noise_case(100, 52, C=1, seed=15),
    "blob64": lambda: blob_case(),
    "blob_nonsquare": lambda: blob_case(80, R=8, height=48),
    "species96x64": lambda: species_case(),
    "species_s075": lambda: species_case(seed=2, distribution_size=0.75),
    "species_s05_n3": lambda: species_case(seed=3, distribution_size=0.5, n=3.0),
    "species_n2p5_beta2": lambda: species_case(seed=4, n=2.5, beta_a=2.0),
    "point_mode": lambda: species_case(seed=5, distribution_size=1e-6),
}


@pytest.mark.parametrize("name", sorted(TRANSPORT_CASES))
def test_transport_bit_exact(name):
    cfg, st = TRANSPORT_CASES[name]()
    orc = O.OraclePropagator(cfg)
    aff = orc.affinity(st)
    exp = orc.transport(st, aff)
    with fl.CudaPropagator(cfg) as p:
        got = p.debug_transport(st, aff)
    if name == "point_mode":
        # nearest-cell deposits: same cells, summation order may differ
        np.testing.assert_allclose(got, exp, rtol=1e-6, atol=1e-7)
    else:
        assert np.array_equal(got, exp), f"max diff {np.abs(got - exp).max()}"


def test_transport_wide_gather_radius():
    """Heavy weights push the flow bound past the fast-path radius: the
    general gather must still match (bit-exact: the order is preserved)."""
    cfg, st = species_case(seed=6)
    for k in cfg["kernels"]:
        k["weight"] = 12.0
    orc = O.OraclePropagator(cfg)
    aff = orc.affinity(st)
    exp = orc.transport(st, aff)
    with fl.CudaPropagator(cfg) as p:
        got = p.debug_transport(st, aff)
    assert np.array_equal(got, exp), f"max diff {np.abs(got - exp).max()}"


def test_transport_tiny_world_wraps_many_times():
    """8x8 torus with large flows: sources wrap several times (reintegration.rs:418-442)."""
    cfg, st = species_case(W=8, H=8, C=1, R=2, seed=7, patches=2, patch=4)
    cfg["kernels"][0]["weight"] = 40.0
    orc = O.OraclePropagator(cfg)
    aff = orc.affinity(st)
    exp = orc.transport(st, aff)
    with fl.CudaPropagator(cfg) as p:
        got = p.debug_transport(st, aff)
    np.testing.assert_allclose(got, exp, rtol=1e-6, atol=1e-7)
    assert abs(got.sum(dtype=np.float64) - st.sum(dtype=np.float64)) < 1e-5


AFF_CASES = {
    "blob64_R10": lambda: blob_case(),
    "species80x60_untemplated": lambda: species_case(80, 60, C=2, R=7, seed=14),
    "blob256_R13": lambda: blob_case(256, R=13, steps_in=2),
    "species96x64": lambda: species_case(),
    "species128_R15": lambda: species_case(128, 128, R=15, seed=8),
}


@pytest.mark.parametrize("mode", [fl.CONV_DIRECT, fl.CONV_FFT])
@pytest.mark.parametrize("name", sorted(AFF_CASES))
def test_affinity_close_to_fp64(name, mode):
    cfg, st = AFF_CASES[name]()
    exp32 = O.OraclePropagator(cfg).affinity(st)
    exp64 = O.OraclePropagator(cfg, f64=True).affinity(st.astype(np.float64))
    with fl.CudaPropagator(cfg, conv_mode=mode) as p:
        p.write_state(st)
        got = p.debug_affinity()
    err_orc = np.abs(exp32 - exp64).max()
    err_gpu = np.abs(got - exp64).max()
    assert err_gpu <= AFF_FACTOR * err_orc + AFF_ABS, (err_gpu, err_orc)


STEP_CASES = {
    "blob64": lambda: blob_case(steps_in=0),
    "blob256_R13": lambda: blob_case(256, R=13, steps_in=0),
    "species96x64": lambda: species_case(),
    "species128_R15": lambda: species_case(128, 128, R=15, seed=9),
}


@pytest.mark.parametrize("mode", [fl.CONV_DIRECT, fl.CONV_FFT])
@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_step_parity_1_and_10(name, mode):
    cfg, st = STEP_CASES[name]()
    orc = O.OraclePropagator(cfg)
    with fl.CudaPropagator(cfg, conv_mode=mode) as p:
        state = fl.SimulationState(st, cfg["width"], cfg["height"])
        p.step(state)
        e1 = orc.run(st, 1)
        assert np.abs(state.channels - e1).max() <= STEP1_TOL
        p.run(state, 9)
        e10 = orc.run(e1, 9)
        assert np.abs(state.channels - e10).max() <= STEP10_TOL
        assert state.step == 10
        assert state.time == pytest.approx(np.float32(0.2) * 10, rel=1e-6)


def test_run_graph_matches_eager_steps():
    """run(n) replays a captured graph; it must equal n single steps bit for bit."""
    cfg, st = species_case(seed=10)
    with fl.CudaPropagator(cfg) as p1, fl.CudaPropagator(cfg) as p2:
        p1.write_state(st)
        p2.write_state(st)
        p1.run_device(37)
        for _ in range(37):
            nat_step(p2)
        assert np.array_equal(p1.read_state(), p2.read_state())
        assert p1.info().step == 37


def test_step_host_matches_device_steps():
    """flp_step_host (copy in, steps, copy out, one synchronisation) equals
    write_state + run + read_state bit for bit and advances the clock; works on
    pinned and on pageable host memory."""
    cfg, st = species_case(seed=14)
    with fl.CudaPropagator(cfg) as p1, fl.CudaPropagator(cfg) as p2:
        p1.write_state(st)
        p1.run_device(3)
        ref3 = p1.read_state()
        p1.run_device(1)
        ref4 = p1.read_state()
        pin = fl.propagator.PinnedBuffer(st.shape)
        pin.array[...] = st
        t, n = p2.step_host(pin.array, steps=3, time=0.0, step=0)
        assert np.array_equal(pin.array, ref3)
        assert n == 3 and t == pytest.approx(float(np.float32(0.2) * 3), rel=1e-6)
        host = np.array(pin.array)
        t, n = p2.step_host(host)
        assert np.array_equal(host, ref4)
        assert n == 4
        with pytest.raises(ValueError):
            p2.step_host(host.astype(np.float64))


def _one_source_case():
    """C=2 with every kernel reading channel 0: channel 1 is no source."""
    rng = np.random.default_rng(15)
    ks = [wl.kernel(0, t, wl.random_rings(rng, 1, 2), weight=0.7, mu=0.18, sigma=0.03) for t in (0, 1)]
    cfg = wl.config(128, 64, 2, ks, kernel_radius=9)
    st = np.zeros((2, 128 * 64), np.float32)
    st[:, 20 * 128 + 30: 20 * 128 + 60] = rng.random((2, 30), dtype=np.float32)
    st[:, 40 * 128 + 70: 40 * 128 + 100] = rng.random((2, 30), dtype=np.float32)
    return cfg, st


@pytest.mark.parametrize("case", ["species96x64", "one_source", "width80"])
@pytest.mark.parametrize("steps", [1, 2, 3, 11])
def test_step_host_pinned_matches_pageable_and_device(case, steps):
    """On the FFT path a pinned host state is read by the first step's row
    transforms directly (widths with a warp-synchronous row transform; channels
    that no kernel reads are copied); pageable memory, and widths without that
    transform, are copied in.  Every form gives the device-resident run's bits
    and the same clock."""
    if case == "species96x64":
        cfg, st = species_case(seed=16)
    elif case == "one_source":
        cfg, st = _one_source_case()
    else:
        cfg, st = species_case(W=80, H=48, C=2, seed=17)
    with fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p1, fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p2:
        p1.write_state(st)
        p1.run_device(steps)
        ref = p1.read_state()
        pin = fl.propagator.PinnedBuffer(st.shape)
        pin.array[...] = st
        t, n = p2.step_host(pin.array, steps=steps, time=0.0, step=0)
        assert np.array_equal(pin.array, ref)
        assert n == steps and t == pytest.approx(p1.info().time, rel=0, abs=0)
        assert np.array_equal(p2.read_state(), ref)  # the device state follows the host one
        host = st.copy()
        p2.step_host(host, steps=steps, time=0.0, step=0)
        assert np.array_equal(host, ref)
        # a further call continues from the host buffer, not from the device state
        pin.array[...] = st
        p2.step_host(pin.array, steps=steps, time=0.0, step=0)
        assert np.array_equal(pin.array, ref)


def nat_step(p):
    from autoverse_b200 import _native as nat
    nat.check(nat.lib().flp_step(p._h))


def test_mass_conservation_fp64():
    """Reference bound: < 0.1% over 100 steps (propagator.rs:561-592).  The
    engine is measured with the FP64 compensated reduction."""
    cfg, st = blob_case(steps_in=0)
    with fl.CudaPropagator(cfg) as p:
        p.write_state(st)
        m0 = p.total_mass()
        p.run_device(100)
        p.synchronize()
        m1 = p.total_mass()
    assert abs(m1 - m0) / m0 < 1e-4
    assert abs(m0 - st.astype(np.float64).sum()) / m0 < 1e-12


def test_total_mass_f32_matches_reference_order():
    cfg, st = species_case(seed=11)
    with fl.CudaPropagator(cfg) as p:
        p.write_state(st)
        assert p.total_mass_f32() == O.total_mass(st.reshape(-1)) or \
            p.total_mass_f32() == sum_channels_f32(st)


def sum_channels_f32(st):
    tot = np.float32(0)
    for ch in st:
        tot = np.float32(tot + O.total_mass(np.ascontiguousarray(ch)))
    return float(tot)


def test_autotuner_picks_a_mode_and_caches_per_shape():
    """The first handle of a shape measures (convolution path, FFT pass CTA
    shapes, gather rows per thread); a second handle of the same shape takes
    the cached choices."""
    cfg, st = species_case(W=160, H=96, C=2, seed=12)  # a shape no other test uses
    with fl.CudaPropagator(cfg) as p:
        p.write_state(st)
        t1 = p.tuning()
        assert p.conv_mode in (fl.CONV_DIRECT, fl.CONV_FFT)
        assert not t1["cached"]
    with fl.CudaPropagator(cfg) as q:
        q.write_state(st)
        t2 = q.tuning()
        assert t2["cached"]
        assert {k: v for k, v in t2.items() if k != "cached"} == {k: v for k, v in t1.items() if k != "cached"}


TUNING_VARIANTS = [
    {},
    {"wpc_r2c": 4}, {"wpc_cols": 4}, {"share_cols": 0}, {"share_cols": 0, "wpc_cols": 4}, {"wpc_c2r": 4},
    {"gather_gby": 2},
    {"wpc_r2c": 4, "wpc_cols": 4, "share_cols": 0, "wpc_c2r": 4, "gather_gby": 2},
]


@pytest.mark.parametrize("shape", [(512, 512, 3), (96, 64, 2), (384, 192, 1)])
def test_every_tuning_choice_gives_the_same_bits(shape):
    """Every launch choice the tuner can make computes the same bits (the
    FFT passes transform each line the same way whatever the CTA shape; the
    gather sums each destination in the same order)."""
    W, H, C = shape
    cfg, st = species_case(W=W, H=H, C=C, R=9, seed=15)
    base = dict(conv_mode=fl.CONV_FFT, wpc_r2c=8, wpc_cols=8, share_cols=1, wpc_c2r=8, gather_gby=1)
    ref = None
    with fl.CudaPropagator(cfg) as p:
        for v in TUNING_VARIANTS:
            p.set_tuning(**dict(base, **v))
            p.write_state(st)
            p.run_device(4)
            got = p.read_state()
            if ref is None:
                ref = got
            assert np.array_equal(got, ref), v


def test_profile_run_reports_stages():
    cfg, st = species_case(seed=13)
    with fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p:
        p.write_state(st)
        prof = p.profile_run(3, flush_l2=True)
    assert set(prof["stages"]) == {"fft_rows_r2c", "fft_cols_conv", "fft_rows_c2r_growth", "flow_2d", "gather_2d"}
    assert prof["step_ms"] > 0
