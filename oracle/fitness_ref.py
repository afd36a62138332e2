"""Fitness evaluation restated in numpy — TEST INFRASTRUCTURE ONLY.

A restatement of the reference's FitnessEvaluator (src/compute/evolution/
fitness.rs:26-88) and its metrics (fitness.rs:91-520) over the f32 oracle
propagator.  Sums run sequentially in f32, in the reference's row-major order
(np.cumsum accumulates one element at a time), so the metric values follow the
reference's own rounding.  Only the test suite and the benchmark's CPU leg use
it, as the checker of the engine's batched fitness evaluation.

Configs are the reference's JSON: a fitness config
{"metrics": [{"metric": {"type": "Persistence"}, "weight": 1.0}, ...],
 "normalize": true} and an evaluation config {"steps": 200, "warmup_steps": 0,
"sample_interval": 10} (schema/evolution.rs:273-314, 479-514).
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

F = np.float32


def seqsum(a) -> np.float32:
    """f32 sum, one element after another (Iterator::sum over f32)."""
    a = np.asarray(a, dtype=F).reshape(-1)
    return F(0.0) if a.size == 0 else np.cumsum(a, dtype=F)[-1]


def channel_sum(state: np.ndarray) -> np.ndarray:
    """SimulationState::channel_sum (propagator.rs:109-120): per cell, channels added in order."""
    s = np.zeros(state.shape[1], dtype=F)
    for ch in state:
        s = (s + ch.astype(F)).astype(F)
    return s


def total_mass(state: np.ndarray) -> np.float32:
    """total_mass_all_channels (reintegration.rs:221-228)."""
    return seqsum([seqsum(ch) for ch in state])


def center_of_mass(grid: np.ndarray, w: int, h: int):
    """fitness.rs:195-215."""
    g = np.asarray(grid, dtype=F)
    idx = np.flatnonzero(g > 0)
    m = g[idx]
    xs = (idx % w).astype(F)
    ys = (idx // w).astype(F)
    tot = seqsum(m)
    cx = seqsum((xs * m).astype(F))
    cy = seqsum((ys * m).astype(F))
    if tot > F(1e-6):
        return F(cx / tot), F(cy / tot)
    return F(F(w) / F(2.0)), F(F(h) / F(2.0))


def radius(grid: np.ndarray, cx, cy, w: int, h: int) -> np.float32:
    """fitness.rs:218-240."""
    g = np.asarray(grid, dtype=F)
    idx = np.flatnonzero(g > 0)
    m = g[idx]
    dx = ((idx % w).astype(F) - F(cx)).astype(F)
    dy = ((idx // w).astype(F) - F(cy)).astype(F)
    tot = seqsum(m)
    mom = seqsum((m * ((dx * dx).astype(F) + (dy * dy).astype(F)).astype(F)).astype(F))
    if tot > F(1e-6):
        return F(math.sqrt(F(mom / tot)))
    return F(0.0)


def similarity(a, b) -> np.float32:
    """fitness.rs:337-350: normalised dot product."""
    a = np.asarray(a, dtype=F)
    b = np.asarray(b, dtype=F)
    if a.size != b.size:
        return F(0.0)
    dot = seqsum((a * b).astype(F))
    na = F(math.sqrt(seqsum((a * a).astype(F))))
    nb = F(math.sqrt(seqsum((b * b).astype(F))))
    if na > F(1e-6) and nb > F(1e-6):
        return F(dot / F(na * nb))
    return F(0.0)


class Trajectory:
    """EvaluationTrajectory (fitness.rs:96-176)."""

    def __init__(self, state: np.ndarray, w: int, h: int):
        self.w, self.h = w, h
        snap = channel_sum(state)
        cx, cy = center_of_mass(snap, w, h)
        self.initial_mass = total_mass(state)
        self.initial_center = (cx, cy)
        self.initial_radius = radius(snap, cx, cy, w, h)
        self.initial_snapshot = snap
        self.centers, self.radii, self.masses, self.maxes, self.actives, self.snapshots = [], [], [], [], [], []

    def record(self, state: np.ndarray, step: int) -> None:
        s = channel_sum(state)
        cx, cy = center_of_mass(s, self.w, self.h)
        self.centers.append((cx, cy))
        self.radii.append(radius(s, cx, cy, self.w, self.h))
        self.masses.append(seqsum(s))
        self.maxes.append(F(max(0.0, float(s.max()))) if s.size else F(0.0))
        self.actives.append(int(np.count_nonzero(s > F(1e-6))))
        self.snapshots.append((step, s))

    def behavior(self) -> dict:
        """to_behavior_stats (fitness.rs:158-185)."""
        disp = F(0.0)
        if len(self.centers) >= 2:
            (x0, y0), (x1, y1) = self.centers[0], self.centers[-1]
            disp = F(math.sqrt(F(F(F(x1 - x0) ** 2) + F(F(y1 - y0) ** 2))))
        return {"final_mass": self.masses[-1] if self.masses else F(0.0), "initial_mass": self.initial_mass,
                "center_of_mass_trajectory": list(self.centers), "total_displacement": disp,
                "radius_over_time": list(self.radii), "final_radius": self.radii[-1] if self.radii else F(0.0),
                "active_cells": self.actives[-1] if self.actives else 0,
                "max_activation": F(max([0.0] + [float(m) for m in self.maxes]))}


# ---- metrics (fitness.rs:243-520) -------------------------------------------

def persistence(t: Trajectory) -> np.float32:
    if t.initial_mass < F(1e-6):
        return F(0.0)
    final_mass = t.masses[-1] if t.masses else F(0.0)
    ratio = F(final_mass / t.initial_mass)
    final_max = t.maxes[-1] if t.maxes else F(0.0)
    active = t.actives[-1] if t.actives else 1
    conc = F(final_max / F(final_mass / F(active))) if final_mass > F(1e-6) else F(0.0)
    return F(min(max(F(F(ratio * F(min(conc, F(10.0)))) / F(10.0)), 0.0), 1.0))


def compactness(t: Trajectory, w: int, h: int) -> np.float32:
    final_radius = t.radii[-1] if t.radii else F(np.finfo(np.float32).max)
    max_radius = F(F(min(w, h)) / F(2.0))
    return F(min(max(F(F(1.0) - F(final_radius / max_radius)), 0.0), 1.0))


def locomotion(t: Trajectory) -> np.float32:
    if len(t.centers) < 2:
        return F(0.0)
    (x0, y0), (x1, y1) = t.centers[0], t.centers[-1]
    disp = F(math.sqrt(F(F(F(x1 - x0) ** 2) + F(F(y1 - y0) ** 2))))
    maxd = F(math.sqrt(F(t.w ** 2 + t.h ** 2)))
    return F(min(max(F(disp / maxd), 0.0), 1.0))


def periodicity(t: Trajectory, period: int, tolerance: float) -> np.float32:
    for step, snap in t.snapshots:
        if step == period:
            sim = similarity(t.initial_snapshot, snap)
            if sim > F(F(1.0) - F(tolerance)):
                return sim
    best = F(0.0)
    for step, snap in t.snapshots:
        if step > 0:
            best = F(max(best, similarity(t.initial_snapshot, snap)))
    return best


def complexity(state: np.ndarray, w: int, h: int) -> np.float32:
    s = channel_sum(state)
    mean = F(seqsum(s) / F(s.size))
    if mean < F(1e-6):
        return F(0.0)
    d = (s - mean).astype(F)
    var = F(seqsum((d * d).astype(F)) / F(s.size))
    g = s.reshape(h, w)
    terms = np.zeros((h, w, 2), dtype=F)  # per cell: x term, then y term
    terms[:, 1:, 0] = np.abs((g[:, 1:] - g[:, :-1]).astype(F))
    terms[1:, :, 1] = np.abs((g[1:, :] - g[:-1, :]).astype(F))
    gsum = seqsum(terms.reshape(-1))  # zero terms (x = 0 or y = 0) leave the sum unchanged
    gmean = F(gsum / F(2 * s.size))
    return F(min(F(F(F(math.sqrt(var)) + gmean) / F(2.0)), F(1.0)))


def mass_concentration(state: np.ndarray) -> np.float32:
    s = channel_sum(state)
    mean = F(seqsum(s) / F(s.size))
    mx = F(max(0.0, float(s.max())))
    if mean < F(1e-6):
        return F(0.0)
    return F(min(F(F(mx / mean) / F(100.0)), F(1.0)))


def glider(t: Trajectory, state: np.ndarray, w: int, h: int, min_displacement: float) -> np.float32:
    loc = locomotion(t)
    comp = compactness(t, w, h)
    disp = F(0.0)
    if len(t.centers) >= 2:
        (x0, y0), (x1, y1) = t.centers[0], t.centers[-1]
        disp = F(math.sqrt(F(F(F(x1 - x0) ** 2) + F(F(y1 - y0) ** 2))))
    if disp < F(min_displacement):
        return F(0.0)
    if len(t.radii) >= 2:
        r = np.asarray(t.radii, dtype=F)
        mean_r = F(seqsum(r) / F(r.size))
        dv = (r - mean_r).astype(F)
        var = F(seqsum((dv * dv).astype(F)) / F(r.size))
        cv = F(F(math.sqrt(var)) / F(max(mean_r, F(1e-6))))
        cons = F(min(max(F(F(1.0) - cv), 0.0), 1.0))
    else:
        cons = F(0.5)
    return F(F(F(F(loc * comp) * cons)) * persistence(t))


def oscillator(t: Trajectory, max_period: int, threshold: float) -> np.float32:
    best = F(0.0)
    for period in range(1, max_period + 1):
        for i, (si, ai) in enumerate(t.snapshots):
            for sj, aj in t.snapshots[i + 1:]:
                if sj - si == period:
                    sim = similarity(ai, aj)
                    if sim > F(threshold):
                        score = F(sim * F(F(1.0) - F(F(F(period) / F(max_period)) * F(0.5))))
                        best = F(max(best, score))
    return best


def stability(t: Trajectory, state: np.ndarray) -> np.float32:
    s = channel_sum(state)
    neg = int(np.count_nonzero(s < 0))
    neg_pen = F(min(F(F(neg) / F(s.size)), F(1.0)))
    mx = F(max(0.0, float(s.max())))
    ext = F(F(mx - F(10.0)) / mx) if mx > F(10.0) else F(0.0)
    final_mass = t.masses[-1] if t.masses else F(0.0)
    err = F(abs(F(F(final_mass - t.initial_mass) / t.initial_mass))) if t.initial_mass > F(1e-6) else F(0.0)
    return F(min(max(F(F(F(F(1.0) - neg_pen) - ext) - err), 0.0), 1.0))


def metric_score(metric: dict, t: Trajectory, state: np.ndarray, w: int, h: int) -> np.float32:
    kind = metric["type"]
    if kind == "Persistence":
        return persistence(t)
    if kind == "Compactness":
        return compactness(t, w, h)
    if kind == "Locomotion":
        return locomotion(t)
    if kind == "Periodicity":
        return periodicity(t, int(metric["period"]), float(metric["tolerance"]))
    if kind == "Complexity":
        return complexity(state, w, h)
    if kind == "MassConcentration":
        return mass_concentration(state)
    if kind == "GliderScore":
        return glider(t, state, w, h, float(metric["min_displacement"]))
    if kind == "OscillatorScore":
        return oscillator(t, int(metric["max_period"]), float(metric["threshold"]))
    if kind == "Stability":
        return stability(t, state)
    return F(0.0)  # Custom: scored outside the evaluator


def combine(metrics: list, scores: list, normalize: bool) -> np.float32:
    """Weighted mean of the scores (fitness.rs:66-82); normalisation clamps to [0, 1]."""
    vals = [F(min(max(s, 0.0), 1.0)) if normalize else F(s) for s in scores]
    weights = [F(m["weight"]) for m in metrics]
    total_w = seqsum(weights)
    num = seqsum([F(v * w) for v, w in zip(vals, weights)])
    return F(num / F(max(total_w, F(1e-6))))


def evaluate(sim_config: dict, seed: dict, fitness: dict, evaluation: dict):
    """FitnessEvaluator::evaluate over the f32 oracle: (fitness, [scores], behavior)."""
    cfg = O.normalize_config(sim_config)
    w, h = cfg["width"], cfg["height"]
    prop = O.OraclePropagator(cfg)
    state = O.seed_generate(seed, cfg)
    t = Trajectory(state, w, h)
    warm = int(evaluation.get("warmup_steps", 0))
    if warm:
        state = prop.run(state, warm)
    t.record(state, 0)
    interval = max(int(evaluation.get("sample_interval", 10)), 1)
    for step in range(1, int(evaluation.get("steps", 200)) + 1):
        state = prop.run(state, 1)
        if step % interval == 0:
            t.record(state, step)
    metrics = fitness.get("metrics", [])
    scores = [metric_score(m["metric"], t, state, w, h) for m in metrics]
    return combine(metrics, scores, bool(fitness.get("normalize", True))), scores, t.behavior()
