"""FLWA animation files: the oracle's restatement of the reference's writer
and the package's player, against the reference's own tests
(src/animation/format.rs:222-325, recorder.rs:233-372, player.rs:243-428).
CPU only."""
import numpy as np
import pytest

import autoverse_b200 as fl
from oracle import animation_ref as A
from oracle import oracle as O


def test_header_roundtrip():
    b = A.header_bytes(64, 48, 32, 2, 1000, 0.1, compression=A.COMPRESSION_LZ4)
    assert len(b) == A.HEADER_SIZE == 52
    h = A.parse_header(b)
    assert (h["width"], h["height"], h["depth"], h["channels"], h["frame_count"]) == (64, 48, 32, 2, 1000)
    assert abs(h["dt"] - 0.1) < 1e-6 and h["compression"] == A.COMPRESSION_LZ4 and not h["delta_encoding"]


def test_frame_encode_decode():
    data = np.arange(100, dtype=np.float32) * np.float32(0.1)
    enc = A.encode_frame(data)
    assert len(enc) == 400
    assert np.array_equal(A.decode_frame(enc, 100), data)


def test_frame_index_roundtrip():
    b = A.index_bytes(12345678, 8192)
    assert len(b) == A.INDEX_SIZE and np.frombuffer(b, "<u8").tolist() == [12345678, 8192]


def noise_state(W=16, H=16, D=1, C=1):
    cfg = {"width": W, "height": H, "depth": D, "channels": C, "dt": 0.1, "kernel_radius": 4, "kernels": [],
           "flow": {"beta_a": 1.0, "n": 2.0, "distribution_size": 1.0}}
    seed = {"pattern": {"type": "Noise", "channel": 0, "amplitude": 0.5, "seed": 42}}
    return cfg, O.seed_generate(seed, cfg)


def record(tmp_path, name, frames, frame_skip=1, max_frames=0, dims=(16, 16, 1, 1)):
    r = A.Recorder(*dims, 0.1, frame_skip=frame_skip, max_frames=max_frames)
    for f in frames:
        r.record_frame(f)
    data, stats = r.finalize()
    path = tmp_path / name
    path.write_bytes(data)
    return path, stats


def test_recorder_basic(tmp_path):
    _, st = noise_state()
    path, stats = record(tmp_path, "t.flwa", [st] * 10)
    assert stats["frame_count"] == 10 and stats["total_bytes"] == path.stat().st_size > 52


def test_recorder_frame_skip(tmp_path):
    _, st = noise_state()
    _, stats = record(tmp_path, "s.flwa", [st] * 20, frame_skip=5)
    assert stats["frame_count"] == 4


def test_recorder_max_frames(tmp_path):
    _, st = noise_state()
    _, stats = record(tmp_path, "m.flwa", [st] * 100, max_frames=5)
    assert stats["frame_count"] == 5


def test_recorder_3d(tmp_path):
    cfg, _ = noise_state(D=8)
    seed = {"pattern": {"type": "GaussianSphere", "center": [0.5, 0.5, 0.5], "radius": 0.2, "amplitude": 1.0,
                        "channel": 0}}
    st = O.seed_generate(seed, cfg)
    _, stats = record(tmp_path, "3d.flwa", [st], dims=(16, 16, 8, 1))
    assert stats["frame_count"] == 1 and stats["average_frame_size"] >= 16 * 16 * 8 * 4


def test_lz4_refused():
    with pytest.raises(ValueError):
        A.Recorder(16, 16, 1, 1, 0.1, compression=A.COMPRESSION_LZ4)


def test_player_roundtrip_and_iterator(tmp_path):
    _, st = noise_state(C=2)
    frames = [st * np.float32(i + 1) for i in range(5)]
    path, _ = record(tmp_path, "p.flwa", frames, dims=(16, 16, 1, 2))
    with fl.AnimationPlayer(path) as p:
        assert p.frame_count() == 5 and p.dimensions() == (16, 16, 1) and p.channels() == 2
        got = [f.channels for f in p.frames()]
        for g, f in zip(got, frames):
            assert np.array_equal(g, np.asarray(f, np.float32).reshape(2, -1))
        with pytest.raises(IndexError):
            p.read_frame(5)


def test_player_3d_roundtrip(tmp_path):
    cfg, _ = noise_state(D=8)
    st = np.random.default_rng(1).random((1, 16 * 16 * 8), dtype=np.float32)
    path, _ = record(tmp_path, "p3.flwa", [st], dims=(16, 16, 8, 1))
    with fl.AnimationPlayer(path) as p:
        assert p.dimensions() == (16, 16, 8)
        assert np.array_equal(p.read_frame(0).channels, st)
