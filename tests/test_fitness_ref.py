"""The numpy restatement of the reference's fitness evaluator
(oracle/fitness_ref.py) against the reference's own fitness tests
(src/compute/evolution/fitness.rs:522-960), ported with their inputs and
thresholds."""
import numpy as np
import pytest

from oracle import fitness_ref as FR
from oracle import oracle as O

F = np.float32


def cfg64():
    # SimulationConfig { width: 64, height: 64, ..Default::default() } (schema/config.rs defaults)
    return {"width": 64, "height": 64, "depth": 1, "channels": 1, "dt": 0.2, "kernel_radius": 13,
            "kernels": [{"radius": 1.0, "rings": [{"amplitude": 1.0, "distance": 0.5, "width": 0.15}],
                         "weight": 1.0, "mu": 0.15, "sigma": 0.015, "source_channel": 0, "target_channel": 0}],
            "flow": {"beta_a": 1.0, "n": 2.0, "distribution_size": 1.0}}


def blob(r, amp=1.0):
    return {"pattern": {"type": "GaussianBlob", "center": [0.5, 0.5], "radius": r, "amplitude": amp, "channel": 0}}


def traj(w, h, centers, radii, masses):
    """create_test_trajectory (fitness.rs:583-612)."""
    t = FR.Trajectory.__new__(FR.Trajectory)
    t.w, t.h = w, h
    t.initial_mass = F(masses[0] if masses else 1.0)
    t.initial_center = centers[0] if centers else (F(w / 2), F(h / 2))
    t.initial_radius = F(radii[0] if radii else 5.0)
    t.initial_snapshot = np.full(w * h, F(t.initial_mass / F(w * h)), dtype=F)
    t.centers = [(F(x), F(y)) for x, y in centers]
    t.radii = [F(r) for r in radii]
    t.masses = [F(m) for m in masses]
    t.maxes = [F(1.0)] * 10
    t.actives = [100] * 10
    t.snapshots = []
    return t


def test_fitness_evaluator_runs():
    fit = {"metrics": [{"metric": {"type": "Persistence"}, "weight": 1.0},
                       {"metric": {"type": "Compactness"}, "weight": 0.5}], "normalize": True}
    f, scores, beh = FR.evaluate(cfg64(), blob(0.1), fit, {"steps": 10, "sample_interval": 5})
    assert f >= 0.0 and len(scores) == 2 and beh["initial_mass"] > 0.0


def test_center_of_mass():
    assert FR.center_of_mass(np.array([0.0, 0.0, 1.0, 0.0], F), 2, 2) == (0.0, 1.0)


def test_state_similarity():
    a = np.array([1, 0, 0, 1], F)
    c = np.array([0, 1, 1, 0], F)
    assert abs(FR.similarity(a, a) - 1.0) < 1e-6
    assert abs(FR.similarity(a, c)) < 1e-6


def test_locomotion_moving_vs_static():
    s = traj(64, 64, [(32, 32)] * 3, [5.0] * 3, [1.0] * 3)
    m = traj(64, 64, [(32, 32), (40, 40), (50, 50)], [5.0] * 3, [1.0] * 3)
    assert FR.locomotion(m) > FR.locomotion(s)
    assert FR.locomotion(s) < 0.01


def test_compactness_small_vs_diffuse():
    c = cfg64()
    out = []
    for r in (0.05, 0.3):
        st = O.seed_generate(blob(r), c)
        t = FR.Trajectory(st, 64, 64)
        t.record(st, 0)
        out.append(FR.compactness(t, 64, 64))
    assert out[0] > out[1]


def test_persistence_surviving_vs_dissipating():
    s = traj(64, 64, [(32, 32)] * 5, [5.0] * 5, [1.0, 0.98, 0.96, 0.95, 0.95])
    d = traj(64, 64, [(32, 32)] * 5, [5.0, 10.0, 20.0, 40.0, 60.0], [1.0, 0.8, 0.5, 0.2, 0.05])
    assert FR.persistence(s) > FR.persistence(d)


def test_complexity_structured_vs_uniform():
    c = cfg64()
    st = FR.complexity(O.seed_generate(blob(0.1), c), 64, 64)
    un = FR.complexity(O.seed_generate(blob(0.5, 0.1), c), 64, 64)
    assert st > un or st > 0.01


def test_mass_concentration_peaked_vs_flat():
    c = cfg64()
    assert FR.mass_concentration(O.seed_generate(blob(0.03), c)) > FR.mass_concentration(O.seed_generate(blob(0.4), c))


def test_glider_score_requires_movement():
    c = cfg64()
    state = O.seed_generate(blob(0.1), c)
    g = traj(64, 64, [(20, 20), (25, 25), (30, 30), (35, 35), (40, 40)], [5.0] * 5, [1.0, 0.98, 0.96, 0.95, 0.94])
    s = traj(64, 64, [(32, 32)] * 5, [5.0] * 5, [1.0, 0.98, 0.96, 0.95, 0.94])
    gs, ss = FR.glider(g, state, 64, 64, 10.0), FR.glider(s, state, 64, 64, 10.0)
    assert gs > ss and ss < 0.01


def test_periodicity_with_repeating_state():
    t = traj(8, 8, [(4, 4)] * 10, [2.0] * 10, [1.0] * 10)
    a = np.array([1.0 if i % 2 == 0 else 0.0 for i in range(64)], F)
    b = np.array([1.0 if i % 2 == 1 else 0.0 for i in range(64)], F)
    t.initial_snapshot = a
    t.snapshots = [(0, a), (5, b), (10, a), (15, b), (20, a)]
    assert FR.periodicity(t, 10, 0.1) > 0.5


def test_oscillator_score_finds_period():
    t = traj(8, 8, [(4, 4)] * 10, [2.0] * 10, [1.0] * 10)
    a = np.array([1.0 if i < 32 else 0.0 for i in range(64)], F)
    b = np.array([1.0 if i >= 32 else 0.0 for i in range(64)], F)
    t.snapshots = [(0, a), (1, b), (2, a), (3, b), (4, a)]
    assert FR.oscillator(t, 10, 0.8) > 0.3


def test_stability_penalizes_negative_values():
    c = cfg64()
    st = O.seed_generate(blob(0.1), c)
    t = FR.Trajectory(st, 64, 64)
    t.record(st, 0)
    assert FR.stability(t, st) >= 0.0


def test_radius_computation():
    g = np.zeros(100, F)
    for y, x in ((3, 3), (3, 7), (7, 3), (7, 7)):
        g[y * 10 + x] = 1.0
    cx, cy = FR.center_of_mass(g, 10, 10)
    assert abs(cx - 5.0) < 0.1 and abs(cy - 5.0) < 0.1
    assert abs(FR.radius(g, cx, cy, 10, 10) - 2.83) < 0.1


def test_sequential_sum_is_sequential():
    # f32 addition order matters: 1e8 + 1 + ... stays 1e8 one element at a time
    assert FR.seqsum([1e8] + [1.0] * 10) == F(1e8)
