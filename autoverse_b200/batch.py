"""Batched worlds: many independent 2D Flow Lenia worlds advanced together.

The reference advances a population by running one ``CpuPropagator`` per
candidate (src/compute/evolution/search.rs:152-172,
src/compute/evolution/fitness.rs:26-88).  ``BatchedPropagator`` holds every
world in pooled device buffers and advances all of them with persistent
kernels that pull (world, tile) items from device work queues; ``run(n)``
replays a captured CUDA graph of the step loop.  Each world gives the same
bits as a single-world ``CudaPropagator`` with the same config.
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Any, Sequence

import numpy as np

from . import _native as nat
from .propagator import SimulationConfig, _to_json


def _load_configs(configs: Sequence[Any]) -> tuple[list[SimulationConfig], list[bytes]]:
    """Each config as a SimulationConfig and as the JSON text passed to the
    engine, which parses and validates it.  A dict is serialised once and kept
    as a shallow copy (the batch reads only its sides and channel count);
    JSON text or a path is parsed once."""
    texts = [_to_json(c) for c in configs]
    cfgs = []
    for c, t in zip(configs, texts):
        d = SimulationConfig(c) if isinstance(c, dict) else SimulationConfig(json.loads(t))
        d.setdefault("depth", 1)
        cfgs.append(d)
    return cfgs, [t.encode() for t in texts]


class BatchedPropagator:
    def __init__(self, configs: Sequence[Any]):
        self.configs, blobs = _load_configs(configs)
        arr = (C.c_char_p * len(blobs))(*blobs)
        h = C.c_void_p()
        nat.check(nat.lib().flp_batch_create(arr, len(blobs), C.byref(h)))
        self._h = h

    def reconfigure(self, configs: Sequence[Any]) -> None:
        """New configs for the same worlds (flp_batch_reconfigure): each world
        keeps its sides, channel count and kernels' (source, target) channel
        pairs; growth, ring, radius, flow and dt parameters may change.  The
        device pools, work queues and step graphs are reused; states are zeroed
        and clocks reset.  Raises FlpError (INVALID_ARGUMENT) when a world's
        layout differs, ConfigError for an invalid config; either way the
        batch is left unchanged."""
        cfgs, blobs = _load_configs(configs)
        arr = (C.c_char_p * len(blobs))(*blobs)
        nat.check(nat.lib().flp_batch_reconfigure(self._h, arr, len(blobs)))
        self.configs = cfgs

    def layout_matches(self, configs: Sequence[Any]) -> bool:
        """Whether reconfigure(configs) keeps every world's layout."""
        if len(configs) != len(self.configs):
            return False
        for old, c in zip(self.configs, (c if isinstance(c, dict) else SimulationConfig.load(c) for c in configs)):
            if (c["width"], c["height"], c.get("depth", 1), c["channels"]) != \
                    (old["width"], old["height"], old.get("depth", 1), old["channels"]):
                return False
            pairs = lambda cfg: [(k.get("source_channel"), k.get("target_channel")) for k in cfg.get("kernels", [])]
            if pairs(c) != pairs(old):
                return False
        return True

    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().flp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self) -> int:
        return len(self.configs)

    def _shape(self, i: int):
        c = self.configs[i]
        return (c.channels, c.width * c.height)

    def write_world(self, i: int, state: np.ndarray) -> None:
        s = np.ascontiguousarray(state, dtype=np.float32)
        nat.check(nat.lib().flp_batch_write_world(self._h, int(i), s.ctypes.data, s.size))

    def load_seed(self, i: int, seed: Any) -> None:
        nat.check(nat.lib().flp_batch_state_from_seed(self._h, int(i), _to_json(seed).encode()))

    def load_seeds(self, seeds: Sequence[Any]) -> None:
        """load_seed for every world at once (None leaves a world as it is)."""
        if len(seeds) != len(self.configs):
            raise ValueError("need one seed entry per world")
        blobs = [None if sd is None else _to_json(sd).encode() for sd in seeds]
        arr = (C.c_char_p * len(blobs))(*blobs)
        nat.check(nat.lib().flp_batch_states_from_seeds(self._h, arr, len(blobs)))

    def read_world(self, i: int) -> np.ndarray:
        out = np.empty(self._shape(i), dtype=np.float32)
        nat.check(nat.lib().flp_batch_read_world(self._h, int(i), out.ctypes.data, out.size, None, None))
        return out

    def run(self, steps: int) -> None:
        nat.check(nat.lib().flp_batch_run(self._h, C.c_uint64(int(steps))))

    def synchronize(self, timeout_ms: float | None = None) -> None:
        if timeout_ms is None:
            nat.check(nat.lib().flp_batch_synchronize(self._h))
        else:
            nat.check(nat.lib().flp_batch_synchronize_for(self._h, float(timeout_ms)))

    def total_mass(self) -> np.ndarray:
        out = np.empty(len(self), dtype=np.float64)
        nat.check(nat.lib().flp_batch_total_mass(self._h, out.ctypes.data, len(self)))
        return out

    def info(self) -> dict:
        n = C.c_int()
        cc = C.c_size_t()
        cells = C.c_size_t()
        nat.check(nat.lib().flp_batch_info(self._h, C.byref(n), C.byref(cc), C.byref(cells)))
        sets = C.c_int()
        kb = C.c_size_t()
        nat.check(nat.lib().flp_batch_kernel_spectra(self._h, C.byref(sets), C.byref(kb)))
        return {"worlds": n.value, "cell_channels": cc.value, "cells": cells.value, "kernel_spectra": sets.value,
                "kernel_spectra_bytes": kb.value}

    def stream(self) -> int:
        return nat.lib().flp_batch_stream(self._h) or 0

    def profile_run(self, steps: int, flush_l2: bool = True, stages: bool = True) -> dict:
        """Run `steps` eager steps with CUDA events between the stages (or,
        with stages=False, around each step only); summed device ms."""
        ms = (C.c_float * 5)()
        step_ms = C.c_float()
        nat.check(nat.lib().flp_batch_profile_run(self._h, int(steps), int(bool(flush_l2)), ms if stages else None,
                                                  C.byref(step_ms)))
        names = ["batch_r2c", "batch_cols", "batch_c2r", "batch_flow", "batch_gather"]
        return {"stages": {n: ms[i] for i, n in enumerate(names)} if stages else {}, "step_ms": step_ms.value,
                "steps": int(steps), "launches_per_step": 5}

    # ---- trajectory statistics (fitness evaluation) -------------------------
    NSTAT = 12
    STAT_NAMES = ("total", "positive", "cx", "cy", "radius", "max", "active", "negative", "mean", "variance",
                  "gradient_mean", "cells")

    def stats(self) -> np.ndarray:
        """(n_worlds, 12) statistics of each world's channel sum, reduced in FP64
        on the device (flp_batch_stats; columns in STAT_NAMES order)."""
        out = np.empty((len(self), self.NSTAT), dtype=np.float64)
        nat.check(nat.lib().flp_batch_stats(self._h, out.ctypes.data, out.size))
        return out

    def reserve_snapshots(self, n_slots: int) -> None:
        nat.check(nat.lib().flp_batch_reserve_snapshots(self._h, int(n_slots)))

    def snapshot(self, slot: int) -> None:
        """Keep every world's current channel sum in device slot `slot`."""
        nat.check(nat.lib().flp_batch_snapshot(self._h, int(slot)))

    def similarity(self, slot_a: int, slot_b: int) -> np.ndarray:
        """Normalised dot product of two snapshot slots, per world."""
        out = np.empty(len(self), dtype=np.float64)
        nat.check(nat.lib().flp_batch_similarity(self._h, int(slot_a), int(slot_b), out.ctypes.data, out.size))
        return out

