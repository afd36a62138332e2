"""Batched worlds on the GPU: each world of an uneven batch against the
oracle (1e-5 after 1 step, 1e-4 after 10), and bit-equality with the
single-world engine on the same config (same item functions)."""
import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import workloads as wl
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def small_batch(n=10, seed=3):
    return wl.batched_worlds(n, sides=(64, 96, 128), seed=seed)


def test_batch_matches_oracle_per_world():
    worlds = small_batch()
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        states = []
        for i, (cfg, seed) in enumerate(worlds):
            b.load_seed(i, seed)
            states.append(O.seed_generate(seed, cfg))
        b.run(1)
        for i, (cfg, _) in enumerate(worlds):
            exp = O.OraclePropagator(cfg).run(states[i], 1)
            assert np.abs(b.read_world(i) - exp).max() <= 1e-5, i
        b.run(9)
        for i, (cfg, _) in enumerate(worlds):
            exp = O.OraclePropagator(cfg).run(states[i], 10)
            assert np.abs(b.read_world(i) - exp).max() <= 1e-4, i


def test_batch_bit_equal_to_single_world_engine():
    worlds = small_batch(6, seed=4)
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        for i, (_, seed) in enumerate(worlds):
            b.load_seed(i, seed)
        b.run(19)  # graph replays plus eager steps
        for i, (cfg, seed) in enumerate(worlds):
            with fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p:
                p.load_seed(seed)
                p.run_device(19)
                assert np.array_equal(b.read_world(i), p.read_state()), i


def test_batch_mass_and_info():
    worlds = small_batch(5, seed=5)
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        for i, (_, seed) in enumerate(worlds):
            b.load_seed(i, seed)
        m0 = b.total_mass()
        b.run(40)
        b.synchronize()
        m1 = b.total_mass()
        assert np.all(np.abs(m1 - m0) / m0 < 1e-4)
        info = b.info()
        assert info["worlds"] == 5
        assert info["cells"] == sum(c["width"] * c["height"] for c, _ in worlds)


def test_sweep_shares_kernel_spectra_and_keeps_single_world_bits():
    """A parameter sweep (one grid, one set of kernel shapes, per-world growth,
    flow and dt) stores one kernel-spectrum set; a world of another grid gets
    its own.  Every world still equals the single-world engine bit for bit."""
    worlds = wl.sweep_worlds(5, side=64, seed=5) + wl.sweep_worlds(1, side=96, seed=5)
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        info = b.info()
        assert info["kernel_spectra"] == 2
        assert info["kernel_spectra_bytes"] == 8 * 4 * (33 * 64 + 49 * 96)
        for i, (_, seed) in enumerate(worlds):
            b.load_seed(i, seed)
        b.run(11)
        for i, (cfg, seed) in enumerate(worlds):
            with fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p:
                p.load_seed(seed)
                p.run_device(11)
                assert np.array_equal(b.read_world(i), p.read_state()), i
    distinct = wl.sweep_worlds(4, side=64, seed=6, distinct_kernels=True)
    with fl.BatchedPropagator([c for c, _ in distinct]) as b:
        assert b.info()["kernel_spectra"] == 4


def test_batch_seeds_in_one_call_match_per_world_loads():
    worlds = small_batch(7, seed=8)
    seeds = [sd for _, sd in worlds]
    with fl.BatchedPropagator([c for c, _ in worlds]) as a, fl.BatchedPropagator([c for c, _ in worlds]) as b:
        for i, sd in enumerate(seeds):
            a.load_seed(i, sd)
        b.load_seeds([sd if i % 3 else None for i, sd in enumerate(seeds)])  # worlds 0, 3, 6 left empty
        for i in range(len(worlds)):
            got = b.read_world(i)
            assert np.array_equal(got, a.read_world(i) if i % 3 else np.zeros_like(got)), i
        b.load_seeds([seeds[i] if i % 3 == 0 else None for i in range(len(seeds))])
        for i in range(len(worlds)):
            assert np.array_equal(b.read_world(i), a.read_world(i)), i


def assert_single_world_bits(b, worlds, steps):
    for i, (cfg, seed) in enumerate(worlds):
        with fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p:
            p.load_seed(seed)
            p.run_device(steps)
            assert np.array_equal(b.read_world(i), p.read_state()), i


def test_reconfigure_keeps_single_world_bits():
    """flp_batch_reconfigure (the next generation of an evolution run): new
    parameters in the same layouts give the single-world engine's bits, with
    the pools and the step graphs of the first generation reused."""
    worlds = small_batch(6, seed=7)
    nxt = wl.mutated_worlds(worlds, 8)
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        b.load_seeds([s for _, s in worlds])
        b.run(18)  # the step graphs of the first generation
        b.reconfigure([c for c, _ in nxt])
        assert np.all(b.total_mass() == 0.0)  # states zeroed
        b.load_seeds([s for _, s in nxt])
        b.run(19)
        assert_single_world_bits(b, nxt, 19)


def test_reconfigure_grows_and_shrinks_the_spectrum_pool():
    """A sweep (one shared spectrum set) reconfigured to distinct kernels needs
    a larger pool, which drops the captured graphs; back to shared kernels
    reuses it."""
    shared = wl.sweep_worlds(4, side=64, channels=1, R=9, seed=9)
    distinct = wl.sweep_worlds(4, side=64, channels=1, R=9, seed=10, distinct_kernels=True)
    with fl.BatchedPropagator([c for c, _ in shared]) as b:
        assert b.info()["kernel_spectra"] == 1
        b.load_seeds([s for _, s in shared])
        b.run(16)
        b.reconfigure([c for c, _ in distinct])
        assert b.info()["kernel_spectra"] == 4
        b.load_seeds([s for _, s in distinct])
        b.run(17)
        assert_single_world_bits(b, distinct, 17)
        b.reconfigure([c for c, _ in shared])
        assert b.info()["kernel_spectra"] == 1
        b.load_seeds([s for _, s in shared])
        b.run(17)
        assert_single_world_bits(b, shared, 17)


def test_reconfigure_refuses_other_layouts_and_bad_configs_unchanged():
    import json
    worlds = small_batch(3, seed=11)
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        wider = json.loads(json.dumps([c for c, _ in worlds]))
        wider[1]["width"] = 2 * wider[1]["width"]
        with pytest.raises(fl._native.FlpError) as e:
            b.reconfigure(wider)
        assert e.value.code == -2 and "keeps its sides" in str(e.value)
        bad = json.loads(json.dumps([c for c, _ in worlds]))
        bad[2]["dt"] = -0.1
        with pytest.raises(fl._native.ConfigError):
            b.reconfigure(bad)
        with pytest.raises(fl._native.FlpError):
            b.reconfigure([c for c, _ in worlds][:2])
        # the batch still runs its original worlds
        b.load_seeds([s for _, s in worlds])
        b.run(5)
        assert_single_world_bits(b, worlds, 5)


def test_noise_filled_worlds_bit_equal_to_single_world_engine():
    """Mass in every cell of every world: the batched gather (two rows per
    thread) and the single-world gather (one row) take different torus-edge
    paths and must give the same bits."""
    worlds = small_batch(6, seed=21)
    rng = np.random.default_rng(22)
    states = [(0.05 + 0.1 * rng.random((c["channels"], c["width"] * c["height"]))).astype(np.float32)
              for c, _ in worlds]
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        for i, st in enumerate(states):
            b.write_world(i, st)
        b.run(3)
        for i, (cfg, _) in enumerate(worlds):
            with fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p:
                p.write_state(states[i])
                p.run_device(3)
                assert np.array_equal(b.read_world(i), p.read_state()), i

