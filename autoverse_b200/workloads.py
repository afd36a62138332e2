"""Seeded synthetic workloads with the shapes, sizes and value distributions of
the engine's benchmark configurations.  All randomness comes from
``numpy.random.default_rng(seed)``; the default seed is 0x5EED.

* ``single_blob``     — 2D, 1 channel, one ring kernel, Gaussian-blob seed
                        (256x256, R=13 as benchmarked; any size for tests).
* ``multispecies``    — 2D, C channels, all C*C source->target kernels with
                        1-3 random rings each, uniform-noise patches.
* ``batched_worlds``  — many independent 2D worlds of uneven sides, channels,
                        radii and parameters (see batch.py).
* ``sweep_worlds``    — a growth/flow parameter sweep: worlds of one grid that
                        share their kernel shapes.
* ``mutated_worlds``  — the next generation of a population: the same world
                        layouts with new kernel, growth and flow parameters.
* ``sphere3d``        — 3D, one spherical-shell kernel, Gaussian-sphere seed.
"""
from __future__ import annotations

import json

import numpy as np

DEFAULT_SEED = 0x5EED

RING = {"amplitude": 1.0, "distance": 0.5, "width": 0.15}


def kernel(src=0, tgt=0, rings=None, weight=1.0, mu=0.15, sigma=0.015, radius=1.0):
    return {"radius": radius, "rings": rings or [dict(RING)], "weight": weight, "mu": mu, "sigma": sigma,
            "source_channel": src, "target_channel": tgt}


def config(width, height, channels, kernels, dt=0.2, kernel_radius=13, depth=1, beta_a=1.0, n=2.0, s=1.0):
    return {"width": width, "height": height, "depth": depth, "channels": channels, "dt": dt,
            "kernel_radius": kernel_radius, "kernels": kernels,
            "flow": {"beta_a": beta_a, "n": n, "distribution_size": s}}


def single_blob(size=256, R=13, mu=0.15, sigma=0.015, dt=0.2, blob_radius=0.1, height=None):
    cfg = config(size, height or size, 1, [kernel(mu=mu, sigma=sigma)], dt=dt, kernel_radius=R)
    seed = {"pattern": {"type": "GaussianBlob", "center": [0.5, 0.5], "radius": blob_radius, "amplitude": 1.0,
                        "channel": 0}}
    return cfg, seed


def random_rings(rng, lo=1, hi=3):
    return [{"amplitude": float(rng.uniform(0.2, 1.0)), "distance": float(rng.uniform(0.2, 0.9)),
             "width": float(rng.uniform(0.05, 0.2))} for _ in range(int(rng.integers(lo, hi + 1)))]


def multispecies(size=512, channels=3, R=15, patches=20, patch=40, seed=DEFAULT_SEED, height=None, dt=0.2):
    """C channels, K = C*C kernels (every source->target pair), random rings and
    growth parameters; state = `patches` uniform-noise squares per channel on
    zeros (later patches overwrite earlier ones)."""
    rng = np.random.default_rng(seed)
    H = height or size
    ks = []
    for src in range(channels):
        for tgt in range(channels):
            ks.append(kernel(src, tgt, random_rings(rng), weight=float(rng.uniform(0.3, 1.0)),
                             mu=float(rng.uniform(0.1, 0.3)), sigma=float(rng.uniform(0.01, 0.05))))
    cfg = config(size, H, channels, ks, dt=dt, kernel_radius=R)
    state = np.zeros((channels, H, size), dtype=np.float32)
    for c in range(channels):
        for _ in range(patches):
            x0 = int(rng.integers(0, size - patch + 1)) if size > patch else 0
            y0 = int(rng.integers(0, H - patch + 1)) if H > patch else 0
            ph, pw = min(patch, H), min(patch, size)
            state[c, y0:y0 + ph, x0:x0 + pw] = rng.uniform(0.0, 1.0, (ph, pw)).astype(np.float32)
    return cfg, state.reshape(channels, -1)


def patches_as_custom_seed(state: np.ndarray, width: int, height: int) -> dict:
    """The same state expressed in the reference's seed schema (Pattern::Custom,
    src/schema/seed.rs:126-129); only non-zero cells are listed."""
    vals = []
    C = state.shape[0]
    st = state.reshape(C, height, width)
    for c in range(C):
        ys, xs = np.nonzero(st[c])
        vals.extend([int(x), int(y), c, float(st[c, y, x])] for y, x in zip(ys, xs))
    return {"pattern": {"type": "Custom", "values": vals}}


BATCH_SIDES = (64, 96, 128, 192, 256, 384, 512)


def batched_worlds(n=4096, sides=BATCH_SIDES, seed=DEFAULT_SEED):
    """Independent 2D worlds for batched runs: width and height drawn
    independently from `sides`, 1-2 channels, K = C*C kernels (every
    source->target pair) with 1-2 rings of the multispecies distributions,
    kernel_radius ~ U{8..20}, mu ~ U(0.1,0.3), sigma ~ U(0.01,0.05),
    dt ~ U(0.1,0.3), weight ~ U(0.3,1); one Gaussian blob per channel with
    radius ~ U(0.05,0.15).  Returns [(config, seed), ...]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        W = int(rng.choice(sides))
        H = int(rng.choice(sides))
        C = int(rng.integers(1, 3))
        R = int(rng.integers(8, 21))
        ks = []
        for src in range(C):
            for tgt in range(C):
                ks.append(kernel(src, tgt, random_rings(rng, 1, 2), weight=float(rng.uniform(0.3, 1.0)),
                                 mu=float(rng.uniform(0.1, 0.3)), sigma=float(rng.uniform(0.01, 0.05))))
        cfg = config(W, H, C, ks, dt=float(rng.uniform(0.1, 0.3)), kernel_radius=R)
        blobs = [{"center": [float(rng.uniform(0.3, 0.7)), float(rng.uniform(0.3, 0.7))],
                  "radius": float(rng.uniform(0.05, 0.15)), "amplitude": 1.0, "channel": c} for c in range(C)]
        out.append((cfg, {"pattern": {"type": "MultiBlob", "blobs": blobs}}))
    return out


def mutated_worlds(worlds, seed=DEFAULT_SEED):
    """The next generation of an evolution run over `worlds`: the same world
    layouts (sides, channels, kernels' channel pairs) with new rings (1-2),
    mu ~ U(0.1,0.3), sigma ~ U(0.01,0.05), weight ~ U(0.3,1), kernel_radius
    ~ U{8..20}, dt ~ U(0.1,0.3) and beta_a ~ U(0.5,2); seeds unchanged."""
    rng = np.random.default_rng(seed)
    out = []
    for cfg, sd in worlds:
        c = json.loads(json.dumps(cfg))
        c["kernel_radius"] = int(rng.integers(8, 21))
        c["dt"] = float(rng.uniform(0.1, 0.3))
        c["flow"]["beta_a"] = float(rng.uniform(0.5, 2.0))
        for k in c["kernels"]:
            k["rings"] = random_rings(rng, 1, 2)
            k["mu"] = float(rng.uniform(0.1, 0.3))
            k["sigma"] = float(rng.uniform(0.01, 0.05))
            k["weight"] = float(rng.uniform(0.3, 1.0))
        out.append((c, sd))
    return out


def sweep_worlds(n=1024, side=256, channels=2, R=13, seed=DEFAULT_SEED, distinct_kernels=False):
    """A growth/flow parameter sweep: n worlds of one grid sharing one set of
    K = C*C kernel shapes (rings and radius drawn once), each with its own
    weights, mu ~ U(0.1,0.3), sigma ~ U(0.01,0.05), dt ~ U(0.1,0.3) and
    beta_a ~ U(0.5,2); one Gaussian blob per channel.  distinct_kernels gives
    every world its own ring draw instead (the same per-step work, no shared
    kernel spectra).  Returns [(config, seed), ...]."""
    rng = np.random.default_rng(seed)
    shapes = [random_rings(rng, 1, 2) for _ in range(channels * channels)]
    out = []
    for _ in range(n):
        rings = [random_rings(rng, 1, 2) for _ in shapes] if distinct_kernels else shapes
        ks = [kernel(i // channels, i % channels, rings[i], weight=float(rng.uniform(0.3, 1.0)),
                     mu=float(rng.uniform(0.1, 0.3)), sigma=float(rng.uniform(0.01, 0.05)))
              for i in range(channels * channels)]
        cfg = config(side, side, channels, ks, dt=float(rng.uniform(0.1, 0.3)), kernel_radius=R,
                     beta_a=float(rng.uniform(0.5, 2.0)))
        blobs = [{"center": [float(rng.uniform(0.3, 0.7)), float(rng.uniform(0.3, 0.7))],
                  "radius": float(rng.uniform(0.05, 0.15)), "amplitude": 1.0, "channel": c} for c in range(channels)]
        out.append((cfg, {"pattern": {"type": "MultiBlob", "blobs": blobs}}))
    return out


def sphere3d(size=128, R=10, mu=0.15, sigma=0.017, radius=0.12, dt=0.2):
    cfg = config(size, size, 1, [kernel(mu=mu, sigma=sigma)], dt=dt, kernel_radius=R, depth=size)
    seed = {"pattern": {"type": "GaussianSphere", "center": [0.5, 0.5, 0.5], "radius": radius, "amplitude": 1.0,
                        "channel": 0}}
    return cfg, seed



def adjoint_worlds(n=64, size=256, channels=2, R=13, seed=DEFAULT_SEED):
    """Worlds for differentiation: `channels` channels, K = C*C kernels (every
    source->target pair) with 1-3 rings and the multispecies parameter
    distributions, beta_a=1, n=2, s=1, dt=0.2, and a seed of one Gaussian blob
    per channel (centre ~U(0.35,0.65), radius ~U(0.06,0.12)).
    Returns [(config, seed), ...]; the loss target is `shifted(state0)`."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        ks = []
        for src in range(channels):
            for tgt in range(channels):
                ks.append(kernel(src, tgt, random_rings(rng), weight=float(rng.uniform(0.3, 1.0)),
                                 mu=float(rng.uniform(0.1, 0.3)), sigma=float(rng.uniform(0.01, 0.05))))
        cfg = config(size, size, channels, ks, dt=0.2, kernel_radius=R)
        blobs = [{"center": [float(rng.uniform(0.35, 0.65)), float(rng.uniform(0.35, 0.65))],
                  "radius": float(rng.uniform(0.06, 0.12)), "amplitude": 1.0, "channel": c} for c in range(channels)]
        out.append((cfg, {"pattern": {"type": "MultiBlob", "blobs": blobs}}))
    return out


def shifted(state: np.ndarray, width: int, height: int, shift: int = 20) -> np.ndarray:
    """The state moved `shift` cells along +x on the torus (the adjoint loss target)."""
    C = state.shape[0]
    return np.ascontiguousarray(np.roll(state.reshape(C, height, width), shift, axis=2).reshape(C, -1))
