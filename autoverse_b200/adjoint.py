"""Differentiable Flow Lenia: a hand-written adjoint of the 2D step on the GPU.

The reference's propagators run forward only (src/compute/propagator.rs:239-420).
``AdjointBatch`` runs T steps of a batch of same-shape worlds, keeping the
state every k steps, and its ``backward`` turns dL/dA_T into dL/dA_0 and
dL/d(parameters) with the engine's adjoint kernels (no autograd framework).
``FlowLeniaFunction`` wraps the pair in the forward/backward shape of an
autograd Function.

Parameter vector of one world (``param_names``): beta_a, then per kernel
weight, mu, sigma, then per ring amplitude, distance, width.
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Any, Sequence

import numpy as np

from . import _native as nat
from .propagator import SimulationConfig, _to_json


def param_names(config: Any) -> list[str]:
    c = SimulationConfig.load(config)
    out = ["beta_a"]
    for i, k in enumerate(c["kernels"]):
        out += [f"k{i}.weight", f"k{i}.mu", f"k{i}.sigma"]
        for j, _ in enumerate(k["rings"]):
            out += [f"k{i}.r{j}.amplitude", f"k{i}.r{j}.distance", f"k{i}.r{j}.width"]
    return out


class AdjointBatch:
    """Same-shape 2D worlds with a differentiable T-step forward pass."""

    def __init__(self, configs: Sequence[Any]):
        self.configs = [SimulationConfig.load(c) for c in configs]
        blobs = [json.dumps(c).encode() for c in self.configs]
        arr = (C.c_char_p * len(blobs))(*blobs)
        h = C.c_void_p()
        nat.check(nat.lib().flp_adj_create(arr, len(blobs), C.byref(h)))
        self._h = h
        c0 = self.configs[0]
        self.C, self.H, self.W = c0.channels, c0.height, c0.width
        self.n_worlds = len(self.configs)
        counts = []
        for i in range(self.n_worlds):
            n = C.c_int()
            nat.check(nat.lib().flp_adj_param_count(self._h, i, C.byref(n)))
            counts.append(n.value)
        self.param_counts = counts
        self.param_offsets = np.concatenate([[0], np.cumsum(counts)]).astype(int)

    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().flp_adj_destroy(self._h)
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

    @property
    def world_size(self) -> int:
        return self.C * self.H * self.W

    def write_state(self, i: int, state: np.ndarray) -> None:
        a = np.ascontiguousarray(state, dtype=np.float32).reshape(-1)
        nat.check(nat.lib().flp_adj_write_state(self._h, int(i), a.ctypes.data, a.size))

    def load_seed(self, i: int, seed: Any) -> None:
        nat.check(nat.lib().flp_adj_state_from_seed(self._h, int(i), _to_json(seed).encode()))

    def forward(self, steps: int, checkpoint_every: int = 8) -> None:
        nat.check(nat.lib().flp_adj_forward(self._h, int(steps), int(checkpoint_every)))

    def read_final(self, i: int) -> np.ndarray:
        out = np.empty(self.world_size, dtype=np.float32)
        nat.check(nat.lib().flp_adj_read_final(self._h, int(i), out.ctypes.data, out.size))
        return out.reshape(self.C, self.H * self.W)

    def backward(self, dl_dfinal: np.ndarray):
        """dl_dfinal: (n_worlds, C, H*W).  Returns (dL/dA_0 with the same shape,
        [per-world parameter-gradient vectors])."""
        g = np.ascontiguousarray(dl_dfinal, dtype=np.float32).reshape(-1)
        gi = np.empty_like(g)
        gp = np.empty(int(self.param_offsets[-1]), dtype=np.float64)
        nat.check(nat.lib().flp_adj_backward(self._h, g.ctypes.data, g.size, gi.ctypes.data, gi.size,
                                             gp.ctypes.data, gp.size))
        grads = [gp[self.param_offsets[i]:self.param_offsets[i + 1]].copy() for i in range(self.n_worlds)]
        return gi.reshape(self.n_worlds, self.C, self.H * self.W), grads

    def timings(self) -> tuple[float, float]:
        """Device milliseconds of the last forward and backward passes."""
        f, b = C.c_float(), C.c_float()
        nat.check(nat.lib().flp_adj_timings(self._h, C.byref(f), C.byref(b)))
        return f.value, b.value


class FlowLeniaFunction:
    """forward(ctx, batch, states, steps, k) -> final states; backward(ctx,
    dL/d(final)) -> (dL/d(states), per-world parameter gradients), in the
    shape of an autograd Function (``ctx`` is any attribute holder)."""

    @staticmethod
    def forward(ctx, batch: AdjointBatch, states: np.ndarray, steps: int, checkpoint_every: int = 8) -> np.ndarray:
        for i in range(batch.n_worlds):
            batch.write_state(i, states[i])
        batch.forward(steps, checkpoint_every)
        ctx.batch = batch
        return np.stack([batch.read_final(i) for i in range(batch.n_worlds)])

    @staticmethod
    def backward(ctx, grad_final: np.ndarray):
        return ctx.batch.backward(grad_final)
