"""Restatement of the reference's FLWA animation writer -- TEST INFRASTRUCTURE ONLY.

Follows src/animation/format.rs:1-220 (header, frame index, little-endian f32
frame encoding) and src/animation/recorder.rs:56-200 (frame skip, maximum
frame count, index table at the end, header rewritten with the final frame
count).  Only the test suite imports it, to check the CUDA engine's recorder
byte for byte; the product writes its files itself.

LZ4 compression sits behind the reference's optional `lz4` cargo feature
(lz4_flex, absent from the reference tree); without it the reference refuses
LZ4 (recorder.rs:62-69), and so does this restatement.
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = b"FLWA"          # format.rs:6
VERSION = 1              # format.rs:9
HEADER_SIZE = 52         # format.rs:78-81
INDEX_SIZE = 16          # format.rs:147
COMPRESSION_NONE, COMPRESSION_LZ4 = 0, 1


def flags_to_u16(compression: int, delta: bool = False) -> int:
    """AnimationFlags::to_u16 (format.rs:40-47)."""
    return (compression & 0x0F) | ((1 << 4) if delta else 0)


def header_bytes(width: int, height: int, depth: int, channels: int, frame_count: int, dt: float,
                 compression: int = COMPRESSION_NONE, delta: bool = False) -> bytes:
    """AnimationHeader::write_to (format.rs:95-108): magic, version, flags,
    width, height, depth, channels (u32), frame count (u64), dt (f32),
    16 reserved zero bytes, all little-endian."""
    return (MAGIC + struct.pack("<HHIIIIQf", VERSION, flags_to_u16(compression, delta), width, height, depth,
                                channels, frame_count, float(np.float32(dt))) + bytes(16))


def parse_header(b: bytes) -> dict:
    """AnimationHeader::read_from (format.rs:111-160)."""
    if b[:4] != MAGIC:
        raise ValueError("Invalid FLWA magic bytes")
    version, flags, w, h, d, c, n, dt = struct.unpack("<HHIIIIQf", b[4:36])
    if version != VERSION:
        raise ValueError(f"Unsupported FLWA version: {version}")
    return {"width": w, "height": h, "depth": d, "channels": c, "frame_count": n, "dt": dt,
            "compression": flags & 0x0F, "delta_encoding": bool(flags & (1 << 4))}


def index_bytes(offset: int, size: int) -> bytes:
    """FrameIndex::write_to (format.rs:149-153)."""
    return struct.pack("<QQ", offset, size)


def encode_frame(data: np.ndarray) -> bytes:
    """encode_frame (format.rs:171-178): f32 values, little-endian."""
    return np.ascontiguousarray(data, dtype="<f4").tobytes()


def decode_frame(b: bytes, n: int) -> np.ndarray:
    """decode_frame (format.rs:180-198)."""
    if len(b) != 4 * n:
        raise ValueError(f"Frame size mismatch: {len(b)} bytes vs {n} floats")
    return np.frombuffer(b, dtype="<f4").astype(np.float32)


class Recorder:
    """AnimationRecorder (recorder.rs:56-200) writing into memory."""

    def __init__(self, width: int, height: int, depth: int, channels: int, dt: float, frame_skip: int = 1,
                 max_frames: int = 0, compression: int = COMPRESSION_NONE):
        if compression == COMPRESSION_LZ4:
            raise ValueError("LZ4 compression requested but 'lz4' feature is not enabled")
        self.dims = (width, height, depth, channels)
        self.dt = dt
        self.frame_skip, self.max_frames = frame_skip, max_frames
        self.body = bytearray(header_bytes(width, height, depth, channels, 0, dt))
        self.index: list[tuple[int, int]] = []
        self.step_counter = 0

    def record_frame(self, channels: np.ndarray) -> bool:
        """record_frame (recorder.rs:109-166): the skip counter counts calls;
        a frame is written on every frame_skip-th call until max_frames."""
        self.step_counter += 1
        if self.step_counter < self.frame_skip:
            return False
        self.step_counter = 0
        if self.max_frames > 0 and len(self.index) >= self.max_frames:
            return False
        data = encode_frame(np.asarray(channels, dtype=np.float32).reshape(-1))
        self.index.append((len(self.body), len(data)))
        self.body += data
        return True

    def finalize(self) -> tuple[bytes, dict]:
        """finalize (recorder.rs:171-200): index table, then the header again
        with the frame count; returns the file and AnimationStats."""
        index_offset = len(self.body)
        out = bytearray(self.body)
        for off, size in self.index:
            out += index_bytes(off, size)
        n = len(self.index)
        out[:HEADER_SIZE] = header_bytes(*self.dims, n, self.dt)
        stats = {"frame_count": n, "total_bytes": index_offset + n * INDEX_SIZE,
                 "average_frame_size": (index_offset - HEADER_SIZE) // n if n else 0}
        return bytes(out), stats
