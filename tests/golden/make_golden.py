"""Generates the golden fixtures in this directory from the CPU oracle (the
C restatement of CpuPropagator / CpuPropagator3D, f32 build, one thread).

Each ``<case>.npz`` holds, for one reduced-size instance of a benchmark
configuration (same parameters and seeds, smaller sides):
  config  JSON text of the SimulationConfig (reference schema)
  state0  initial state, C x N f32 ([c][z][y][x])
  aff0    affinity U of state0 (growth-weighted kernel sums per target)
  flow0   flow field F of the first step (C x dims x N)
  step1   state after 1 step;  step10  state after 10 steps

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from autoverse_b200 import workloads as wl  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cases():
    cfg, seed = wl.single_blob(64, R=13)  # 256x256 blob world at 64x64
    yield "blob64_R13", cfg, O.seed_generate(seed, cfg)
    cfg, st = wl.multispecies(64, channels=3, R=15, patches=6, patch=16, height=48)
    yield "multispecies64x48_C3_R15", cfg, st
    for i, (cfg, seed) in enumerate(wl.batched_worlds(3, sides=(64, 96))):
        yield f"batch_world{i}", cfg, O.seed_generate(seed, cfg)
    cfg, seed = wl.sphere3d(32, R=10)  # 128^3 sphere world at 32^3
    yield "sphere32_R10", cfg, O.seed_generate(seed, cfg)


def main():
    for name, cfg, st in cases():
        orc = O.OraclePropagator(cfg)
        st = np.ascontiguousarray(st, dtype=np.float32)
        aff = orc.affinity(st)
        s1 = orc.run(st, 1)
        flow = orc.last_flow()
        s10 = orc.run(s1, 9)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, config=json.dumps(cfg), state0=st, aff0=aff, flow0=flow, step1=s1, step10=s10)
        print(f"{name}: {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
