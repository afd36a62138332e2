"""The engine's recorder (flp_rec_*) writes the same FLWA bytes as the
restatement of the reference's writer given the same states: frames are taken
in stream order from the device state while the steps keep running."""
import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import workloads as wl
from oracle import animation_ref as A

pytestmark = pytest.mark.gpu


def expected_file(cfg, st, steps, frame_skip, max_frames):
    W, H, D, C = cfg["width"], cfg["height"], cfg.get("depth", 1), cfg["channels"]
    rec = A.Recorder(W, H, D, C, cfg["dt"], frame_skip=frame_skip, max_frames=max_frames)
    with fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p:
        p.write_state(st)
        for _ in range(steps):
            p.run_device(1)
            rec.record_frame(p.read_state())
    return rec.finalize()


@pytest.mark.parametrize("frame_skip,max_frames", [(1, 0), (3, 0), (2, 4)])
def test_recorder_bytes_match_the_reference_writer(tmp_path, frame_skip, max_frames):
    cfg, st = wl.multispecies(64, channels=2, R=8, patches=4, patch=16, seed=1)
    want, stats_want = expected_file(cfg, st, 12, frame_skip, max_frames)
    path = tmp_path / "gpu.flwa"
    with fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT) as p:
        p.write_state(st)
        rec = fl.AnimationRecorder(path, p, frame_skip=frame_skip, max_frames=max_frames)
        rec.run(12)
        stats = rec.finalize()
    assert path.read_bytes() == want
    assert stats["frame_count"] == stats_want["frame_count"] and stats["total_bytes"] == stats_want["total_bytes"]


def test_recorder_interleaved_with_graph_runs_and_3d(tmp_path):
    cfg, seed = wl.sphere3d(32, R=6)
    path = tmp_path / "s3.flwa"
    states = []
    with fl.CudaPropagator(cfg) as p:
        p.load_seed(seed)
        rec = fl.AnimationRecorder(path, p)
        for n in (16, 1, 3):
            p.run_device(n)  # graph replay and single steps; the frame follows them in stream order
            assert rec.record_frame()
            states.append(p.read_state())
        stats = rec.finalize()
    assert stats["frame_count"] == 3
    with fl.AnimationPlayer(path) as pl:
        assert pl.dimensions() == (32, 32, 32)
        for i, s in enumerate(states):
            assert np.array_equal(pl.read_frame(i).channels, s)


def test_recorder_refuses_lz4(tmp_path):
    cfg, st = wl.multispecies(64, channels=1, R=8, patches=2, patch=16, seed=2)
    with fl.CudaPropagator(cfg) as p:
        with pytest.raises(fl.FlpError):
            fl.AnimationRecorder(tmp_path / "x.flwa", p, compression=1)
