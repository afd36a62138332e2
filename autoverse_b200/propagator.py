"""Python mirror of the reference's propagator surface, backed by the CUDA engine.

``CudaPropagator`` has the surface of ``CpuPropagator`` (src/compute/propagator.rs:155-433):
``CudaPropagator(config)``, ``step(state)``, ``run(state, n)``, ``config``;
``SimulationState`` mirrors src/compute/propagator.rs:15-121 (``from_seed``,
``total_mass``, ``channels`` as ``[channel][z*H*W + y*W + x]`` f32 planes,
``time``, ``step``).  Configs and seeds are the reference's JSON schema, given as
JSON text, a path to a ``.json`` file, or a dict.

The state lives in HBM between calls: ``step``/``run`` upload the host state
only when it changed since the last call and always copy the result back into
``state.channels`` (the reference mutates the caller's state in place).
``run_device`` advances without any host copy.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Any

import numpy as np

from . import _native as nat


def _to_json(obj: Any) -> str:
    if isinstance(obj, dict):
        return json.dumps(obj)
    if isinstance(obj, (str, os.PathLike)) and os.path.exists(str(obj)):
        with open(obj) as f:
            return f.read()
    if isinstance(obj, str):
        return obj
    raise TypeError("config/seed must be a dict, JSON text or a path")


class SimulationConfig(dict):
    """The reference's SimulationConfig (src/schema/config.rs:14-35) as a dict."""

    @classmethod
    def load(cls, obj: Any) -> "SimulationConfig":
        d = json.loads(_to_json(obj))
        d.setdefault("depth", 1)
        return cls(d)

    @property
    def width(self) -> int:
        return self["width"]

    @property
    def height(self) -> int:
        return self["height"]

    @property
    def depth(self) -> int:
        return self.get("depth", 1)

    @property
    def channels(self) -> int:
        return self["channels"]

    def is_3d(self) -> bool:
        return self.depth > 1

    def grid_size(self) -> int:
        return self.width * self.height * self.depth


class SimulationState:
    """Host-side state, layout of src/compute/propagator.rs:19-32."""

    def __init__(self, channels: np.ndarray, width: int, height: int, depth: int = 1, time: float = 0.0,
                 step: int = 0):
        self.channels = np.ascontiguousarray(channels, dtype=np.float32).reshape(-1, width * height * depth)
        self.width, self.height, self.depth = width, height, depth
        self.time = float(np.float32(time))
        self.step = int(step)
        self._version = 0

    @classmethod
    def from_seed(cls, seed: Any, config: Any) -> "SimulationState":
        """SimulationState::from_seed (propagator.rs:36-59) via the engine's seed generator."""
        cfg = SimulationConfig.load(config)
        n = cfg.channels * cfg.grid_size()
        out = np.zeros(n, dtype=np.float32)
        nat.check(nat.lib().flp_seed_generate(json.dumps(cfg).encode(), _to_json(seed).encode(),
                                              out.ctypes.data, n))
        return cls(out.reshape(cfg.channels, -1), cfg.width, cfg.height, cfg.depth)

    def is_3d(self) -> bool:
        return self.depth > 1

    def grid_size(self) -> int:
        return self.width * self.height * self.depth

    def total_mass(self) -> float:
        """The reference's naive f32 sum (reintegration.rs:221-228), channel by channel."""
        total = np.float32(0.0)
        for ch in self.channels:
            total = np.float32(total + _seq_sum_f32(ch))
        return float(total)

    def channel_sum(self) -> np.ndarray:
        s = np.zeros(self.grid_size(), dtype=np.float32)
        for ch in self.channels:
            s += ch
        return s


class PinnedBuffer:
    """Page-locked host memory (flp_host_alloc) exposed as a numpy array."""

    def __init__(self, shape, dtype=np.float32):
        self.nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        ptr = C.c_void_p()
        nat.check(nat.lib().flp_host_alloc(self.nbytes, C.byref(ptr)))
        self._ptr = ptr
        buf = (C.c_char * self.nbytes).from_address(ptr.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def __del__(self):
        try:
            if getattr(self, "_ptr", None):
                self.array = None
                nat.lib().flp_host_free(self._ptr)
                self._ptr = None
        except Exception:
            pass


def _seq_sum_f32(x: np.ndarray) -> np.float32:
    """Sequential f32 accumulation (Rust `iter().sum()` order)."""
    acc = np.float32(0.0)
    # chunked cumulative sum keeps the sequential f32 order
    for chunk in np.array_split(np.ascontiguousarray(x, dtype=np.float32), max(1, x.size // 65536)):
        c = np.cumsum(np.concatenate([[acc], chunk]).astype(np.float32), dtype=np.float32)
        acc = c[-1]
    return acc


class CudaPropagator:
    """CpuPropagator's surface on the B200 engine (one world per handle)."""

    def __init__(self, config: Any, conv_mode: int = nat.CONV_AUTO):
        self._config = SimulationConfig.load(config)
        h = C.c_void_p()
        nat.check(nat.lib().flp_create(json.dumps(self._config).encode(), C.byref(h)))
        self._h = h
        self._bound_state: tuple[int, int] | None = None
        if conv_mode != nat.CONV_AUTO:
            self.set_conv_mode(conv_mode)

    # -- lifecycle ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().flp_destroy(self._h)
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

    # -- reference surface ---------------------------------------------------
    def config(self) -> SimulationConfig:
        return self._config

    def step(self, state: SimulationState) -> None:
        self.run(state, 1)

    def run(self, state: SimulationState, steps: int) -> None:
        self.upload(state)
        self.run_device(steps)
        self.download(state)

    # -- device-resident extensions -----------------------------------------
    def upload(self, state: SimulationState) -> None:
        key = (id(state), state._version)
        if self._bound_state == key:
            return
        ch = np.ascontiguousarray(state.channels, dtype=np.float32)
        nat.check(nat.lib().flp_write_state(self._h, ch.ctypes.data, ch.size, C.c_float(state.time),
                                            C.c_uint64(state.step)))
        self._bound_state = key

    def download(self, state: SimulationState) -> None:
        out = np.empty_like(state.channels)
        t = C.c_float()
        s = C.c_uint64()
        nat.check(nat.lib().flp_read_state(self._h, out.ctypes.data, out.size, C.byref(t), C.byref(s)))
        state.channels = out
        state.time = t.value
        state.step = s.value
        state._version += 1
        self._bound_state = (id(state), state._version)

    def load_seed(self, seed: Any) -> None:
        nat.check(nat.lib().flp_state_from_seed(self._h, _to_json(seed).encode()))
        self._bound_state = None

    def run_device(self, steps: int) -> None:
        nat.check(nat.lib().flp_run(self._h, C.c_uint64(int(steps))))

    def synchronize(self, timeout_ms: float | None = None) -> None:
        """Wait for the handle's stream; with timeout_ms, at most that long
        (FlpError with code TIMEOUT when work is still pending)."""
        if timeout_ms is None:
            nat.check(nat.lib().flp_synchronize(self._h))
        else:
            nat.check(nat.lib().flp_synchronize_for(self._h, float(timeout_ms)))

    def step_host(self, channels: np.ndarray, steps: int = 1, time: float | None = None,
                  step: int | None = None) -> tuple[float, int]:
        """Advance a state held in host memory in place (flp_step_host): in,
        `steps` steps, copy back, one synchronisation.  `channels` must be a
        C-contiguous float32 array of channels*cells values; with a
        PinnedBuffer's array the copy back is a DMA transfer and, on the 2D FFT
        path, the first step's row transforms read the state straight from the
        pinned buffer (pageable memory is copied in).  Returns the advanced
        (time, step)."""
        if channels.dtype != np.float32 or not channels.flags["C_CONTIGUOUS"] or not channels.flags["WRITEABLE"]:
            raise ValueError("channels must be a writeable C-contiguous float32 array")
        if time is None or step is None:
            i = self.info()
            time = i.time if time is None else time
            step = i.step if step is None else step
        t, s = C.c_float(time), C.c_uint64(step)
        nat.check(nat.lib().flp_step_host(self._h, channels.ctypes.data, channels.size, C.byref(t), C.byref(s),
                                          C.c_uint64(int(steps))))
        self._bound_state = None
        return t.value, s.value

    def read_state(self) -> np.ndarray:
        info = self.info()
        out = np.empty((info.channels, info.width * info.height * info.depth), dtype=np.float32)
        nat.check(nat.lib().flp_read_state(self._h, out.ctypes.data, out.size, None, None))
        return out

    def write_state(self, channels: np.ndarray, time: float = 0.0, step: int = 0) -> None:
        ch = np.ascontiguousarray(channels, dtype=np.float32)
        nat.check(nat.lib().flp_write_state(self._h, ch.ctypes.data, ch.size, C.c_float(time), C.c_uint64(step)))
        self._bound_state = None

    def total_mass(self) -> float:
        """FP64 compensated sum on the device."""
        out = C.c_double()
        nat.check(nat.lib().flp_total_mass(self._h, C.byref(out)))
        return out.value

    def total_mass_f32(self) -> float:
        out = C.c_float()
        nat.check(nat.lib().flp_total_mass_f32(self._h, C.byref(out)))
        return out.value

    def info(self) -> nat.Info:
        i = nat.Info()
        nat.check(nat.lib().flp_get_info(self._h, C.byref(i)))
        return i

    TUNING_FIELDS = ("conv_mode", "wpc_r2c", "wpc_cols", "share_cols", "wpc_c2r", "gather_gby")

    def tuning(self) -> dict:
        """The autotuner's launch choices for this world's shape (run on first
        use, cached per shape for the process); ``cached`` is True when they
        came from an earlier handle of the same shape."""
        buf = (C.c_int32 * 7)()
        nat.check(nat.lib().flp_get_tuning(self._h, buf, 7))
        out = dict(zip(self.TUNING_FIELDS, list(buf)[:6]))
        out["cached"] = bool(buf[6])
        return out

    def set_tuning(self, **choice) -> None:
        """Force launch choices (any of TUNING_FIELDS; the others keep their
        current values).  No choice changes the results."""
        cur = self.tuning()
        cur.update(choice)
        buf = (C.c_int32 * 6)(*[int(cur[k]) for k in self.TUNING_FIELDS])
        nat.check(nat.lib().flp_set_tuning(self._h, buf, 6))

    def set_conv_mode(self, mode: int) -> None:
        nat.check(nat.lib().flp_set_conv_mode(self._h, int(mode)))

    @property
    def conv_mode(self) -> int:
        return self.info().conv_mode

    def stream(self) -> int:
        return nat.lib().flp_stream(self._h) or 0

    def profile_run(self, steps: int, flush_l2: bool = True, stages: bool = True) -> dict:
        """Run `steps` eager steps with CUDA events around every kernel (or,
        with stages=False, around every step only); returns summed device
        milliseconds per stage and per step (flp_profile_run)."""
        ms = (C.c_float * 16)()
        n = C.c_int()
        names = C.create_string_buffer(512)
        step_ms = C.c_float()
        nat.check(nat.lib().flp_profile_run(self._h, int(steps), int(bool(flush_l2)), ms if stages else None, 16,
                                            C.byref(n), names, 512, C.byref(step_ms)))
        stage_names = names.value.decode().split(",")
        return {"stages": {stage_names[i]: ms[i] for i in range(n.value)} if stages else {},
                "step_ms": step_ms.value, "steps": int(steps), "launches_per_step": n.value}

    def debug_affinity(self) -> np.ndarray:
        info = self.info()
        out = np.empty((info.channels, info.width * info.height * info.depth), dtype=np.float32)
        nat.check(nat.lib().flp_debug_affinity(self._h, out.ctypes.data, out.size))
        return out

    def debug_transport(self, state: np.ndarray, aff: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(state, dtype=np.float32)
        a = np.ascontiguousarray(aff, dtype=np.float32)
        out = np.empty_like(s)
        nat.check(nat.lib().flp_debug_transport(self._h, s.ctypes.data, a.ctypes.data, out.ctypes.data, s.size))
        return out
