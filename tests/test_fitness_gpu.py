"""Population fitness on the batched engine (autoverse_b200/fitness.py)
against the restatement of the reference's FitnessEvaluator over the CPU
oracle (oracle/fitness_ref.py), candidate by candidate, for every built-in
metric.  Device statistics are FP64 sums and the reference's are f32, and
the trajectories agree to the step tolerance, so scores are compared to
2e-3 and behaviour statistics to 1e-4 relative."""
import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import fitness as FT
from autoverse_b200 import workloads as wl
from oracle import fitness_ref as FR

pytestmark = pytest.mark.gpu

ALL_METRICS = {"metrics": [
    {"metric": {"type": "Persistence"}, "weight": 1.0},
    {"metric": {"type": "Compactness"}, "weight": 0.5},
    {"metric": {"type": "Locomotion"}, "weight": 0.7},
    {"metric": {"type": "Periodicity", "period": 10, "tolerance": 0.1}, "weight": 0.3},
    {"metric": {"type": "Complexity"}, "weight": 0.4},
    {"metric": {"type": "MassConcentration"}, "weight": 0.2},
    {"metric": {"type": "GliderScore", "min_displacement": 0.0}, "weight": 0.6},
    {"metric": {"type": "OscillatorScore", "max_period": 10, "threshold": 0.5}, "weight": 0.3},
    {"metric": {"type": "Stability"}, "weight": 0.8},
], "normalize": True}
EVAL = {"steps": 20, "warmup_steps": 3, "sample_interval": 5}


def test_population_matches_reference_evaluator():
    worlds = wl.batched_worlds(6, sides=(64, 96, 128), seed=31)
    got = FT.evaluate_population([c for c, _ in worlds], [s for _, s in worlds], ALL_METRICS, EVAL)
    for (cfg, sd), g in zip(worlds, got):
        f, scores, beh = FR.evaluate(cfg, sd, ALL_METRICS, EVAL)
        for (kind, s, _), e in zip(g["scores"], scores):
            assert abs(s - float(e)) <= 2e-3, (kind, s, float(e))
        assert abs(g["fitness"] - float(f)) <= 2e-3
        assert g["behavior"]["initial_mass"] == pytest.approx(float(beh["initial_mass"]), rel=1e-4)
        assert g["behavior"]["final_mass"] == pytest.approx(float(beh["final_mass"]), rel=1e-4)
        assert g["behavior"]["active_cells"] == pytest.approx(beh["active_cells"], abs=2)
        assert g["behavior"]["final_radius"] == pytest.approx(float(beh["final_radius"]), rel=1e-3, abs=1e-3)


def test_default_configs_and_statistics_shape():
    worlds = wl.batched_worlds(3, sides=(64,), seed=32)
    got = FT.evaluate_population([c for c, _ in worlds], [s for _, s in worlds], evaluation={"steps": 10})
    assert len(got) == 3 and all(len(g["scores"]) == 2 for g in got)
    with fl.BatchedPropagator([c for c, _ in worlds]) as b:
        for i, (_, sd) in enumerate(worlds):
            b.load_seed(i, sd)
        st = b.stats()
        assert st.shape == (3, 12)
        # the statistics add the per-cell f32 channel sums; total_mass adds every channel value
        np.testing.assert_allclose(st[:, 0], b.total_mass(), rtol=1e-6)
        b.reserve_snapshots(2)
        b.snapshot(0)
        b.run(5)
        b.snapshot(1)
        assert np.all(b.similarity(0, 0) > 1 - 1e-12) and np.all(b.similarity(0, 1) <= 1 + 1e-12)


def test_evaluator_reuses_its_batch_across_generations():
    """PopulationEvaluator: a generation with the previous one's layouts is
    evaluated on the same batch (reconfigured), with the scores of a fresh
    evaluation; a generation with other layouts builds a new batch."""
    gen1 = wl.batched_worlds(5, sides=(64, 96), seed=33)
    gen2 = wl.mutated_worlds(gen1, 34)
    gen3 = wl.batched_worlds(5, sides=(128,), seed=35)
    with FT.PopulationEvaluator(ALL_METRICS, EVAL) as ev:
        for gen in (gen1, gen2, gen3):
            got = ev.evaluate([c for c, _ in gen], [s for _, s in gen])
            fresh = FT.evaluate_population([c for c, _ in gen], [s for _, s in gen], ALL_METRICS, EVAL)
            for g, f in zip(got, fresh):
                assert g["fitness"] == f["fitness"] and g["scores"] == f["scores"]
        assert (ev.batches_built, ev.batches_reused) == (2, 1)
