"""Fitness evaluation of a whole population on the batched engine.

The reference evaluates candidates one at a time: each gets its own
CpuPropagator, is run for the evaluation horizon, and its trajectory is
sampled on the host (FitnessEvaluator::evaluate, src/compute/evolution/
fitness.rs:26-88, called per candidate by EvolutionEngine::evaluate_population,
evolution/search.rs:152-172).  Here every candidate is a world of one
BatchedPropagator; the trajectory statistics (mass, centre of mass, radius,
peak, active cells, variance, neighbour differences) are reduced on the device
for all worlds at once, state snapshots stay on the device and their
similarities are reduced there too.  Only a few numbers per world and sample
cross to the host, where the reference's metric formulas (fitness.rs:243-520)
combine them.

``PopulationEvaluator`` keeps its batch from one generation to the next: a
generation with the previous one's world layouts only rebuilds parameters,
kernel spectra and states on the device (flp_batch_reconfigure).

Configs follow the reference's JSON schema (schema/evolution.rs:273-514):
fitness = {"metrics": [{"metric": {"type": "Persistence"}, "weight": 1.0}, ...],
"normalize": true}; evaluation = {"steps": 200, "warmup_steps": 0,
"sample_interval": 10}.  Sums are FP64 on the device, so scores agree with
the reference's f32 host sums to rounding.
"""
from __future__ import annotations

import math
import time
from typing import Any, Sequence

import numpy as np

from ._native import FlpError
from .batch import BatchedPropagator

INVALID_ARGUMENT = -2  # FLP_ERR_INVALID_ARGUMENT: the engine refused a world's new layout

DEFAULT_FITNESS = {"metrics": [{"metric": {"type": "Persistence"}, "weight": 1.0},
                               {"metric": {"type": "Compactness"}, "weight": 0.5}], "normalize": True}
DEFAULT_EVALUATION = {"steps": 200, "warmup_steps": 0, "sample_interval": 10}

T, POS, CX, CY, RAD, MAX, ACT, NEG, MEAN, VAR, GRAD, CELLS = range(12)


def _clamp(v: float, lo: float = 0.0, hi: float = 1.0) -> float:
    return min(max(v, lo), hi)


class _Trajectory:
    """Samples of one world (EvaluationTrajectory, fitness.rs:96-176)."""

    def __init__(self, w: int, h: int, initial: np.ndarray):
        self.w, self.h = w, h
        self.initial_mass = float(initial[T])
        self.initial_center = (float(initial[CX]), float(initial[CY]))
        self.initial_radius = float(initial[RAD])
        self.centers: list = []
        self.radii: list = []
        self.masses: list = []
        self.maxes: list = []
        self.actives: list = []
        self.steps: list = []

    def record(self, st: np.ndarray, step: int) -> None:
        self.centers.append((float(st[CX]), float(st[CY])))
        self.radii.append(float(st[RAD]))
        self.masses.append(float(st[T]))
        self.maxes.append(float(st[MAX]))
        self.actives.append(int(round(st[ACT])))
        self.steps.append(step)

    def displacement(self) -> float:
        if len(self.centers) < 2:
            return 0.0
        (x0, y0), (x1, y1) = self.centers[0], self.centers[-1]
        return math.sqrt((x1 - x0) ** 2 + (y1 - y0) ** 2)

    def behavior(self) -> dict:
        """to_behavior_stats (fitness.rs:158-185)."""
        return {"final_mass": self.masses[-1] if self.masses else 0.0, "initial_mass": self.initial_mass,
                "center_of_mass_trajectory": list(self.centers), "total_displacement": self.displacement(),
                "radius_over_time": list(self.radii), "final_radius": self.radii[-1] if self.radii else 0.0,
                "active_cells": self.actives[-1] if self.actives else 0,
                "max_activation": max([0.0] + self.maxes)}


def _persistence(t: _Trajectory) -> float:
    if t.initial_mass < 1e-6:
        return 0.0
    final_mass = t.masses[-1] if t.masses else 0.0
    conc = t.maxes[-1] / (final_mass / (t.actives[-1] or 1)) if final_mass > 1e-6 else 0.0
    return _clamp(final_mass / t.initial_mass * min(conc, 10.0) / 10.0)


def _compactness(t: _Trajectory) -> float:
    final_radius = t.radii[-1] if t.radii else float(np.finfo(np.float32).max)
    return _clamp(1.0 - final_radius / (min(t.w, t.h) / 2.0))


def _locomotion(t: _Trajectory) -> float:
    if len(t.centers) < 2:
        return 0.0
    return _clamp(t.displacement() / math.sqrt(t.w ** 2 + t.h ** 2))


def _glider(t: _Trajectory, min_displacement: float) -> float:
    if t.displacement() < min_displacement:
        return 0.0
    if len(t.radii) >= 2:
        r = np.asarray(t.radii)
        cons = _clamp(1.0 - math.sqrt(((r - r.mean()) ** 2).mean()) / max(r.mean(), 1e-6))
    else:
        cons = 0.5
    return _locomotion(t) * _compactness(t) * cons * _persistence(t)


def _stability(t: _Trajectory, final: np.ndarray) -> float:
    neg_pen = min(final[NEG] / final[CELLS], 1.0)
    mx = final[MAX]
    ext = (mx - 10.0) / mx if mx > 10.0 else 0.0
    final_mass = t.masses[-1] if t.masses else 0.0
    err = abs((final_mass - t.initial_mass) / t.initial_mass) if t.initial_mass > 1e-6 else 0.0
    return _clamp(1.0 - neg_pen - ext - err)


def _complexity(final: np.ndarray) -> float:
    if final[MEAN] < 1e-6:
        return 0.0
    return min((math.sqrt(final[VAR]) + final[GRAD]) / 2.0, 1.0)


def _concentration(final: np.ndarray) -> float:
    if final[MEAN] < 1e-6:
        return 0.0
    return min(final[MAX] / final[MEAN] / 100.0, 1.0)


class PopulationEvaluator:
    """FitnessEvaluator::evaluate (fitness.rs:26-88) for whole populations,
    generation after generation, on one BatchedPropagator.  A generation whose
    candidates keep the previous generation's world layouts (sides, channels,
    kernels' channel pairs) reuses the batch through reconfigure: its device
    pools, work queues and step graphs, with only the parameters, kernel
    spectra and states rebuilt.  Any other generation builds a new batch."""

    def __init__(self, fitness: dict | None = None, evaluation: dict | None = None):
        self.fitness = fitness or DEFAULT_FITNESS
        self.evaluation = {**DEFAULT_EVALUATION, **(evaluation or {})}
        self._batch: BatchedPropagator | None = None
        self.batches_built = 0
        self.batches_reused = 0

    def close(self) -> None:
        if self._batch is not None:
            self._batch.close()
            self._batch = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def evaluate(self, configs: Sequence[Any], seeds: Sequence[Any], timings: dict | None = None) -> list[dict]:
        """Every (config, seed) pair at once; see evaluate_population."""
        t_start = time.perf_counter()
        reused = False
        if self._batch is not None and self._batch.layout_matches(configs):
            try:
                self._batch.reconfigure(configs)
                reused = True
            except FlpError as e:
                if e.code != INVALID_ARGUMENT:  # not a layout change: a real error
                    raise
        if reused:
            self.batches_reused += 1
        else:
            self.close()
            self._batch = BatchedPropagator(configs)
            self.batches_built += 1
        return _evaluate(self._batch, seeds, self.fitness, self.evaluation, timings, t_start)


def evaluate_population(configs: Sequence[Any], seeds: Sequence[Any], fitness: dict | None = None,
                        evaluation: dict | None = None, timings: dict | None = None) -> list[dict]:
    """FitnessEvaluator::evaluate for every (config, seed) pair at once.
    Returns per candidate {"fitness", "scores": [(type, score, weight)],
    "behavior": {...}} in the reference's shapes.  `timings`, when given,
    receives the wall-clock seconds of the set-up (batch creation and seeds),
    the simulation with its sampling, and the metric evaluation."""
    with PopulationEvaluator(fitness, evaluation) as ev:
        return ev.evaluate(configs, seeds, timings)


def _evaluate(b: BatchedPropagator, seeds: Sequence[Any], fitness: dict, evaluation: dict, timings: dict | None,
              t_start: float) -> list[dict]:
    metrics = fitness.get("metrics", [])
    kinds = [m["metric"]["type"] for m in metrics]
    steps = int(evaluation["steps"])
    warm = int(evaluation.get("warmup_steps", 0))
    interval = max(int(evaluation["sample_interval"]), 1)
    sample_steps = [0] + list(range(interval, steps + 1, interval))
    snaps = any(k in ("Periodicity", "OscillatorScore") for k in kinds)
    b.load_seeds(list(seeds))
    n = len(b)
    if snaps:
        b.reserve_snapshots(1 + len(sample_steps))
        b.snapshot(0)  # the initial state's channel sum
    t_setup = time.perf_counter()
    init = b.stats()
    traj = [_Trajectory(c["width"], c["height"], init[i]) for i, c in enumerate(b.configs)]
    if warm:
        b.run(warm)
    done = 0
    for k, step in enumerate(sample_steps):
        if step > done:
            b.run(step - done)
            done = step
        st = b.stats()
        for i in range(n):
            traj[i].record(st[i], step)
        if snaps:
            b.snapshot(1 + k)
    if done < steps:
        b.run(steps - done)
    final = b.stats()
    t_run = time.perf_counter()
    sim = {}

    def similarity(sa: int, sb: int) -> np.ndarray:
        if (sa, sb) not in sim:
            sim[(sa, sb)] = b.similarity(sa, sb)
        return sim[(sa, sb)]

    results = []
    for i in range(n):
        t = traj[i]
        scores = []
        for m in metrics:
            spec = m["metric"]
            kind = spec["type"]
            if kind == "Persistence":
                v = _persistence(t)
            elif kind == "Compactness":
                v = _compactness(t)
            elif kind == "Locomotion":
                v = _locomotion(t)
            elif kind == "Periodicity":  # fitness.rs:300-334
                v = None
                for k, step in enumerate(sample_steps):
                    if step == int(spec["period"]):
                        s = similarity(0, 1 + k)[i]
                        if s > 1.0 - float(spec["tolerance"]):
                            v = s
                            break
                if v is None:
                    v = max([0.0] + [similarity(0, 1 + k)[i] for k, s in enumerate(sample_steps) if s > 0])
            elif kind == "Complexity":
                v = _complexity(final[i])
            elif kind == "MassConcentration":
                v = _concentration(final[i])
            elif kind == "GliderScore":
                v = _glider(t, float(spec["min_displacement"]))
            elif kind == "OscillatorScore":  # fitness.rs:468-495
                v = 0.0
                maxp, thr = int(spec["max_period"]), float(spec["threshold"])
                for a in range(len(sample_steps)):
                    for c in range(a + 1, len(sample_steps)):
                        period = sample_steps[c] - sample_steps[a]
                        if 1 <= period <= maxp:
                            s = similarity(1 + a, 1 + c)[i]
                            if s > thr:
                                v = max(v, s * (1.0 - period / maxp * 0.5))
            elif kind == "Stability":
                v = _stability(t, final[i])
            else:  # Custom: scored by the caller
                v = 0.0
            scores.append((kind, float(v), float(m["weight"])))
        vals = [_clamp(s) if fitness.get("normalize", True) else s for _, s, _ in scores]
        tw = sum(w for _, _, w in scores)
        f = sum(v * w for v, (_, _, w) in zip(vals, scores)) / max(tw, 1e-6)
        results.append({"fitness": float(f), "scores": scores, "behavior": t.behavior()})
    if timings is not None:
        t_end = time.perf_counter()
        timings.update(setup_s=t_setup - t_start, simulate_s=t_run - t_setup, metrics_s=t_end - t_run)
    return results
