"""Parameter-embedded worlds: Flow Lenia whose cells carry their own growth
and flow parameters, advected and mixed with the mass.

Mirrors the reference's ``EmbeddedState`` / ``EmbeddedPropagator``
(src/compute/embedded_propagator.rs:23-345) on the CUDA engine
(``flp_emb_*`` in include/flowlenia_cuda.h).  Parameter grids are arrays of
shape (channels, height*width, 5) holding CellParams' fields in struct order
(mu, sigma, weight, beta_a, n; src/schema/embedding.rs:20-31).
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Any

import numpy as np

from . import _native as nat
from .propagator import SimulationConfig, _to_json

NPAR = 5
CELL_DEFAULT = (0.15, 0.015, 1.0, 1.0, 2.0)  # CellParams::default (embedding.rs:33-43)


class EmbeddedState:
    """EmbeddedState (embedded_propagator.rs:23-37): channels, parameter grids,
    time and step, on the host."""

    def __init__(self, channels: np.ndarray, params: np.ndarray, width: int, height: int, time: float = 0.0,
                 step: int = 0):
        n = width * height
        self.channels = np.ascontiguousarray(channels, dtype=np.float32).reshape(-1, n)
        self.params = np.ascontiguousarray(params, dtype=np.float32).reshape(self.channels.shape[0], n, NPAR)
        self.width, self.height = width, height
        self.time = float(np.float32(time))
        self.step = int(step)

    @classmethod
    def from_seed(cls, seed: Any, config: Any, params: np.ndarray | None = None) -> "EmbeddedState":
        """EmbeddedState::from_seed / from_seed_with_params (embedded_propagator.rs:39-98)."""
        cfg = SimulationConfig.load(config)
        with EmbeddedPropagator(cfg) as p:
            p.load_seed(seed)
            st = p.read()
        if params is not None:
            st.params = np.ascontiguousarray(params, dtype=np.float32).reshape(st.params.shape).copy()
        return st

    def total_mass(self) -> float:
        return float(self.channels.sum(dtype=np.float64))

    def get_params(self, x: int, y: int, channel: int) -> np.ndarray:
        return self.params[channel, y * self.width + x]


class EmbeddedPropagator:
    """EmbeddedPropagator (embedded_propagator.rs:144-345) on the GPU.

    ``step(state)`` / ``run(state, n)`` follow the reference: the host state
    is copied in, advanced and copied back.  ``load_seed`` / ``write`` /
    ``run_device`` / ``read`` keep the state on the device."""

    def __init__(self, config: Any):
        self._config = SimulationConfig.load(config)
        h = C.c_void_p()
        nat.check(nat.lib().flp_emb_create(json.dumps(self._config).encode(), C.byref(h)))
        self._h = h
        cfg = self._config
        self.width, self.height, self.channels = cfg.width, cfg.height, cfg.channels
        self.cells = cfg.width * cfg.height

    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().flp_emb_destroy(self._h)
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

    def config(self) -> SimulationConfig:
        return self._config

    # -- the reference's surface ----------------------------------------
    def step(self, state: EmbeddedState) -> None:
        self.run(state, 1)

    def run(self, state: EmbeddedState, steps: int) -> None:
        self.write(state)
        self.run_device(steps)
        out = self.read()
        state.channels, state.params, state.time, state.step = out.channels, out.params, out.time, out.step

    # -- device-resident use ---------------------------------------------
    def load_seed(self, seed: Any) -> None:
        nat.check(nat.lib().flp_emb_state_from_seed(self._h, _to_json(seed).encode()))

    def write(self, state: EmbeddedState) -> None:
        ch = np.ascontiguousarray(state.channels, dtype=np.float32)
        pr = np.ascontiguousarray(state.params, dtype=np.float32)
        nat.check(nat.lib().flp_emb_write_state(self._h, ch.ctypes.data, ch.size, pr.ctypes.data, pr.size,
                                                C.c_float(state.time), C.c_uint64(state.step)))

    def write_channels(self, channels: np.ndarray, time: float = 0.0, step: int = 0) -> None:
        ch = np.ascontiguousarray(channels, dtype=np.float32)
        nat.check(nat.lib().flp_emb_write_state(self._h, ch.ctypes.data, ch.size, None, 0, C.c_float(time),
                                                C.c_uint64(step)))

    def read(self) -> EmbeddedState:
        ch = np.empty((self.channels, self.cells), np.float32)
        pr = np.empty((self.channels, self.cells, NPAR), np.float32)
        t = C.c_float()
        s = C.c_uint64()
        nat.check(nat.lib().flp_emb_read_state(self._h, ch.ctypes.data, ch.size, pr.ctypes.data, pr.size,
                                               C.byref(t), C.byref(s)))
        return EmbeddedState(ch, pr, self.width, self.height, t.value, s.value)

    def run_device(self, steps: int) -> None:
        nat.check(nat.lib().flp_emb_run(self._h, C.c_uint64(int(steps))))

    def synchronize(self) -> None:
        nat.check(nat.lib().flp_emb_synchronize(self._h))

    def total_mass(self) -> float:
        out = C.c_double()
        nat.check(nat.lib().flp_emb_total_mass(self._h, C.byref(out)))
        return out.value

    def profile_run(self, steps: int, stages: bool = False) -> dict:
        """Device milliseconds of `steps` steps (CUDA events on the engine's
        stream); with stages, per-kernel totals of eager steps."""
        ms = C.c_float()
        st = (C.c_float * 3)()
        nat.check(nat.lib().flp_emb_profile_run(self._h, C.c_uint64(int(steps)), C.byref(ms),
                                                st if stages else None))
        out = {"step_ms": ms.value}
        if stages:
            out["stages"] = dict(zip(("emb_conv_growth", "emb_flow", "emb_gather"), list(st)))
        return out
