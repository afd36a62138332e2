"""Animation recording and playback in the reference's FLWA format.

``AnimationRecorder`` mirrors src/animation/recorder.rs:56-200 on the CUDA
engine (``flp_rec_*`` in include/flowlenia_cuda.h): frames are taken from a
``CudaPropagator``'s device state without stalling its stream and written by a
background thread.  ``AnimationPlayer`` reads FLWA files as
src/animation/player.rs:26-240 does (header, index table at the end, raw f32
little-endian frames), including files written by the reference.
"""
from __future__ import annotations

import ctypes as C
import os
import struct

import numpy as np

from . import _native as nat
from .propagator import CudaPropagator, SimulationState

HEADER_SIZE = 52
INDEX_SIZE = 16
COMPRESSION_NONE, COMPRESSION_LZ4 = 0, 1


class AnimationRecorder:
    """AnimationRecorder::new(path, config, RecorderConfig) for a propagator:
    ``record_frame()`` takes the propagator's current state (in stream order),
    ``finalize()`` returns AnimationStats as a dict."""

    def __init__(self, path: str | os.PathLike, propagator: CudaPropagator, frame_skip: int = 1,
                 max_frames: int = 0, compression: int = COMPRESSION_NONE):
        h = C.c_void_p()
        nat.check(nat.lib().flp_rec_create(propagator._h, os.fspath(path).encode(), int(compression),
                                           C.c_uint32(int(frame_skip)), C.c_uint64(int(max_frames)),
                                           C.byref(h)))
        self._h = h
        self._prop = propagator  # the handle must outlive the recorder

    def record_frame(self) -> bool:
        rec = C.c_int()
        nat.check(nat.lib().flp_rec_record(self._h, C.byref(rec)))
        return bool(rec.value)

    def run(self, steps: int) -> None:
        """`steps` times: one propagator step, then record_frame()."""
        nat.check(nat.lib().flp_rec_run(self._h, C.c_uint64(int(steps))))

    def frames_written(self) -> int:
        n = C.c_uint64()
        nat.check(nat.lib().flp_rec_frames_written(self._h, C.byref(n)))
        return n.value

    def finalize(self) -> dict:
        if not self._h:
            raise RuntimeError("recorder already finalized")
        n, tot, avg = C.c_uint64(), C.c_uint64(), C.c_uint64()
        h, self._h = self._h, None
        nat.check(nat.lib().flp_rec_finalize(h, C.byref(n), C.byref(tot), C.byref(avg)))
        return {"frame_count": n.value, "total_bytes": tot.value, "average_frame_size": avg.value,
                "compression": "None"}

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                nat.lib().flp_rec_finalize(self._h, None, None, None)
            except Exception:
                pass
            self._h = None


class AnimationPlayer:
    """AnimationPlayer::open (player.rs:36-64) and read_frame (player.rs:101-129)."""

    def __init__(self, path: str | os.PathLike):
        self._f = open(path, "rb")
        head = self._f.read(HEADER_SIZE)
        if len(head) < HEADER_SIZE or head[:4] != b"FLWA":
            raise ValueError("Invalid FLWA magic bytes")
        version, flags, w, h, d, c, n, dt = struct.unpack("<HHIIIIQf", head[4:36])
        if version != 1:
            raise ValueError(f"Unsupported FLWA version: {version}")
        self.header = {"width": w, "height": h, "depth": d, "channels": c, "frame_count": n, "dt": dt,
                       "compression": flags & 0x0F, "delta_encoding": bool(flags & 0x10)}
        if self.header["compression"] != COMPRESSION_NONE:
            raise ValueError("LZ4-compressed animations need the reference's lz4 feature")
        size = self._f.seek(0, os.SEEK_END)
        self._f.seek(size - n * INDEX_SIZE)
        raw = self._f.read(n * INDEX_SIZE)
        self.index = [struct.unpack("<QQ", raw[i * INDEX_SIZE:(i + 1) * INDEX_SIZE]) for i in range(n)]

    def frame_count(self) -> int:
        return self.header["frame_count"]

    def dimensions(self) -> tuple:
        return self.header["width"], self.header["height"], self.header["depth"]

    def channels(self) -> int:
        return self.header["channels"]

    def dt(self) -> float:
        return self.header["dt"]

    def read_frame(self, i: int) -> SimulationState:
        if not 0 <= i < self.frame_count():
            raise IndexError(f"Frame index {i} out of range (max {self.frame_count() - 1})")
        off, size = self.index[i]
        self._f.seek(off)
        data = np.frombuffer(self._f.read(size), dtype="<f4").astype(np.float32)
        w, h, d = self.dimensions()
        return SimulationState(data.reshape(self.channels(), w * h * d), w, h, d)

    def frames(self):
        for i in range(self.frame_count()):
            yield self.read_frame(i)

    def close(self) -> None:
        self._f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
