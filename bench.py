#!/usr/bin/env python
"""Benchmark of the Flow Lenia step engine (one JSON line on stdout, rank 0).

Default workload: 2D multispecies world, 512x512 torus, 3 channels, 9 kernels
(every source->target pair, 1-3 random rings each), R=15, dt=0.2, state = 20
uniform-noise 40x40 patches per channel; seeded synthetic data (seed 0x5EED).

* ``value``: cell-steps/s over exactly K steps, device time from CUDA events
  on the engine's stream, every step preceded by an L2 flush (a write of twice
  the L2 size, outside the timed events), max over ranks.
* ``e2e``: the same metric through the public API with pinned host buffers:
  every step copies the state host->device, steps, and copies it back.
* ``roofline``: the dominant kernel's algorithmic bytes per launch over its
  average event-timed duration, against the measured HBM copy bandwidth.
* ``cpu_baseline``: the CPU oracle (a C restatement of the reference's
  CpuPropagator) on the host cores, on a bounded sample of the same workload.

``--impl reference`` times that CPU implementation alone on the same config
and metric (rank 0; other ranks exit 0).  With ``--gpus N`` under torchrun
every rank runs an independent replica of the world (a single world does not
shard), so ``value`` is N x the per-GPU work over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

WORLD = int(os.environ.get("WORLD_SIZE", "1"))
RANK = int(os.environ.get("RANK", "0"))
LOCAL_RANK = int(os.environ.get("LOCAL_RANK", "0"))
if WORLD > 1 and "CUDA_VISIBLE_DEVICES" not in os.environ:
    os.environ["CUDA_VISIBLE_DEVICES"] = str(LOCAL_RANK)

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload", choices=["multispecies512", "blob256", "sphere128"], default="multispecies512")
    ap.add_argument("--e2e-steps", type=int, default=300)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-flush", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU baseline (profiling runs)")
    ap.add_argument("--tuning", default=None,
                    help="force the FFT launch choices wpc_r2c,wpc_cols,share_cols,wpc_c2r,gather_gby (profiling runs, "
                         "where the tuner's timings are distorted by the profiler); default: the tuner's own")
    ap.add_argument("--conv", choices=["auto", "direct", "fft"], default="auto",
                    help="convolution path (auto = the engine's measured choice)")
    ap.add_argument("--batch-worlds", type=int, default=4096, help="worlds in the batched measurement (0 = skip)")
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--adjoint-worlds", type=int, default=64, help="worlds in the adjoint measurement (0 = skip)")
    ap.add_argument("--adjoint-steps", type=int, default=64)
    ap.add_argument("--adjoint-every", type=int, default=8)
    ap.add_argument("--fitness-candidates", type=int, default=512, help="population of the fitness measurement (0 = skip)")
    ap.add_argument("--embedded-size", type=int, default=256, help="side of the parameter-embedded world (0 = skip)")
    ap.add_argument("--record-steps", type=int, default=400, help="steps of the recording measurement (0 = skip)")
    ap.add_argument("--sweep-worlds", type=int, default=1024, help="worlds of the parameter-sweep measurement (0 = skip)")
    ap.add_argument("--other-steps", type=int, default=1000,
                    help="steps of the blob 256^2 and sphere 128^3 measurements beside the headline (0 = skip)")
    return ap.parse_args()


def seed_state(seed, cfg, engine: bool):
    """Initial state from a seed: the engine's generator (flp_seed_generate)
    on the GPU arm, the oracle's restatement on the reference arm; both give
    the same bits (tests/test_engine_cpu.py)."""
    if engine:
        import autoverse_b200 as fl
        return fl.SimulationState.from_seed(seed, cfg).channels
    from oracle import oracle as O
    return O.seed_generate(seed, cfg)


def workload(name, engine: bool = True):
    from autoverse_b200 import workloads as wl
    if name == "multispecies512":
        cfg, state = wl.multispecies(512, channels=3, R=15)
        desc = {"workload": "multispecies 512x512 torus, 3 channels, 9 kernels (all src->tgt pairs, 1-3 rings), "
                            "R=15, dt=0.2, beta_a=1, n=2, s=1, 20 U(0,1) 40x40 patches per channel",
                "width": 512, "height": 512, "channels": 3, "kernels": 9, "kernel_radius": 15}
    elif name == "sphere128":
        cfg, seed = wl.sphere3d(128)
        state = seed_state(seed, cfg, engine)
        desc = {"workload": "3D sphere 128^3 torus, 1 channel, 1 spherical-shell kernel (ring 1.0/0.5/0.15), R=10, "
                            "mu=0.15, sigma=0.017, dt=0.2, Gaussian sphere r=0.12",
                "width": 128, "height": 128, "depth": 128, "channels": 1, "kernels": 1, "kernel_radius": 10}
    else:
        cfg, seed = wl.single_blob(256)
        state = seed_state(seed, cfg, engine)
        desc = {"workload": "single blob 256x256 torus, 1 channel, 1 kernel (ring 1.0/0.5/0.15), R=13, mu=0.15, "
                            "sigma=0.015, dt=0.2, Gaussian blob r=0.1",
                "width": 256, "height": 256, "channels": 1, "kernels": 1, "kernel_radius": 13}
    return cfg, state, desc


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def stage_bytes(cfg, stage):
    """Algorithmic HBM bytes of one launch of each stage."""
    W, H, C = cfg["width"], cfg["height"], cfg["channels"]
    D = cfg.get("depth", 1)
    K = len(cfg["kernels"])
    N = W * H * D
    nsrc = len({k["source_channel"] for k in cfg["kernels"]})
    spec = (W // 2 + 1) * H * D * 8
    return {
        "fft_x_r2c": nsrc * N * 4 + nsrc * spec,
        "fft_y_fwd": 2 * nsrc * spec,
        "fft_z_conv": (nsrc + 2 * K) * spec,
        "fft_y_inv": 2 * K * spec,
        "fft_x_c2r_growth": K * spec + C * N * 4,
        "flow_3d": 2 * C * N * 4 + 3 * C * N * 4,
        "gather_3d": 4 * C * N * 4 + C * N * 4,
        "fft_rows_r2c": nsrc * N * 4 + nsrc * spec,
        "fft_cols_conv": (nsrc + 2 * K) * spec,
        "fft_rows_c2r_growth": K * spec + C * N * 4,
        "flow_2d": 2 * C * N * 4 + 2 * C * N * 4,
        "gather_2d": 3 * C * N * 4 + C * N * 4,
        "conv_direct_growth_2d": nsrc * N * 4 + C * N * 4,
    }.get(stage)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str):
        self.bus = bus_id.lower()
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 5.0:  # wait for the first sample
                time.sleep(0.05)
                if os.path.getsize(self.file.name) > 0:
                    break
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                bus = parts[0].lower()
                if self.bus and not (bus.endswith(self.bus[-12:]) or self.bus.endswith(bus[-12:])):
                    continue
                rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": num(rows[0][2]),
                "power_w_max": max((num(r[3]) or 0.0) for r in rows), "reasons": reasons, "samples": len(rows)}


def dist_init():
    if WORLD <= 1:
        return None
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", timeout=timedelta(seconds=120))
    return dist


def reduce_max(dist, v: float) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference_run(cfg, state, seconds: float, max_steps: int, warmup: int = 1):
    """The oracle on all host cores: conv parallel over kernels and stencil
    over channels, as the reference's rayon loops (propagator.rs:259-267, 332-371)."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    p = O.OraclePropagator(cfg)
    st = p.run(state, warmup, threads=threads) if warmup else state
    t0 = time.perf_counter()
    n = 0
    while n < max_steps and (n == 0 or (time.perf_counter() - t0) < seconds):
        st = p.run(st, 1, threads=threads)
        n += 1
    dt = time.perf_counter() - t0
    return n, dt, threads


def cpu_worlds_run(worlds, seconds: float):
    """The oracle on all host cores over worlds (one world per thread, as the
    reference's evolution search runs one CpuPropagator per candidate on a
    rayon pool, search.rs:152-172), on the first worlds of the batch: time-
    bounded rounds of one step of every sampled world."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    sample = worlds[:4 * threads]
    props = [O.OraclePropagator(c) for c, _ in sample]
    states = O.run_many(props, [seed_state(sd, c, False) for c, sd in sample], 1, threads)  # warm-up step
    t0 = time.perf_counter()
    rounds = 0
    while rounds == 0 or time.perf_counter() - t0 < seconds:
        states = O.run_many(props, states, 1, threads)
        rounds += 1
    dt = time.perf_counter() - t0
    cells = sum(c["width"] * c["height"] for c, _ in sample)
    return {"value": cells * rounds / dt, "unit": "cell-steps/s", "cores": threads, "kind": "port",
            "sample": f"{len(sample)} of the batch's worlds, {rounds} steps each (time-bounded at {seconds:.0f} s), "
                      "one world per host thread, C restatement of CpuPropagator in f32"}


def measure_batched(args, dist):
    """Batched worlds: `--batch-worlds` independent worlds (sides from
    {64..512} per axis, 1-2 channels, K = C*C, radius 8..20, per-world growth
    and flow parameters), timed as one persistent-kernel step loop; plus the
    batched/plain ratio on 1024 small uneven worlds (sides 64..128), plain
    being one device-resident propagator per world stepped in turn."""
    import autoverse_b200 as fl
    from autoverse_b200 import workloads as wl
    from autoverse_b200 import sharding
    # weak scaling: batch_worlds per GPU; the global list is LPT-partitioned by
    # estimated step cost, every rank deriving the same partition locally
    everything = wl.batched_worlds(args.batch_worlds * WORLD)
    share = sharding.lpt_partition([sharding.world_cost(c) for c, _ in everything], WORLD)[RANK]
    worlds = [everything[i] for i in share]
    b = fl.BatchedPropagator([c for c, _ in worlds])
    for i, (_, sd) in enumerate(worlds):
        b.load_seed(i, sd)
    info = b.info()
    b.profile_run(3, flush_l2=False)
    if dist:
        dist.barrier()
    prof = b.profile_run(args.batch_steps, flush_l2=False, stages=False)
    b.synchronize()
    t = reduce_max(dist, prof["step_ms"] / 1e3)
    sprof = b.profile_run(min(args.batch_steps, 50), flush_l2=False, stages=True)
    stage_ms = {k: v / sprof["steps"] for k, v in sprof["stages"].items()}
    # per-stage algorithmic bytes: the single-world figures summed over the worlds
    names = {"r2c": "fft_rows_r2c", "cols": "fft_cols_conv", "c2r": "fft_rows_c2r_growth", "flow": "flow_2d",
             "gather": "gather_2d"}
    sbytes = {k: sum(stage_bytes(c, names[k.replace("batch_", "")]) for c, _ in worlds)
              for k in stage_ms if k.replace("batch_", "") in names}
    dom = max(stage_ms, key=stage_ms.get)
    peak, peak_kind = hbm_peak()
    step_min = sum(4 * c["width"] * c["height"] * (len({k["source_channel"] for k in c["kernels"]}) +
                                                   4 * c["channels"]) for c, _ in worlds)
    roof = {"bound": "hbm", "kernel": dom, "achieved": sbytes[dom] / (stage_ms[dom] * 1e-3) / 1e9, "peak": peak,
            "unit": "GB/s", "algorithmic_bytes_per_launch": sbytes[dom],
            "per_stage_gbs": {k: sbytes[k] / (stage_ms[k] * 1e-3) / 1e9 for k in sbytes},
            "step_minimum_bytes": step_min,
            "step_minimum_frac": step_min / (t / args.batch_steps) / 1e9 / peak,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else "fallback 6.65 TB/s"}
    roof["frac"] = roof["achieved"] / peak
    out = {"workload": f"{args.batch_worlds} worlds per GPU (LPT-sharded by step cost), sides {{64..512}} per axis, C in {{1,2}}, K=C*C, R~U{{8..20}}, "
                       "mu~U(0.1,0.3), sigma~U(0.01,0.05), dt~U(0.1,0.3), Gaussian-blob seeds",
           "cells_per_gpu": info["cells"], "cell_channels_per_gpu": info["cell_channels"], "steps": args.batch_steps,
           "value": sum(c["width"] * c["height"] for c, _ in everything) * args.batch_steps / t, "unit": "cell-steps/s",
           "ms_per_step": 1e3 * t / args.batch_steps,
           "stage_ms_per_step": stage_ms, "roofline": roof,
           # queue reset, three FFT stages x 7 size classes, the flow's 2 channel-count classes, the gather
           "gpu_launches_per_step": 1 + 3 * 7 + 2 + 1, "l2": "working set above L2 (pooled state and spectra)"}
    b.close()
    if RANK == 0 and not args.skip_cpu:
        out["cpu_baseline"] = cpu_worlds_run(worlds, args.cpu_seconds)
    # batched vs plain on small uneven worlds
    small = wl.batched_worlds(1024, sides=(64, 96, 128), seed=wl.DEFAULT_SEED + 17)
    b = fl.BatchedPropagator([c for c, _ in small])
    for i, (_, sd) in enumerate(small):
        b.load_seed(i, sd)
    steps = 48
    b.run(steps)  # warm-up with the timed step count: every graph either arm replays is built before timing
    b.synchronize()
    t0 = time.perf_counter()
    b.run(steps)
    b.synchronize()
    v_b = b.info()["cells"] * steps / (time.perf_counter() - t0)
    b.close()
    props = []
    for cfg, sd in small[:48]:
        p = fl.CudaPropagator(cfg, conv_mode=fl.CONV_FFT)
        p.load_seed(sd)
        p.run_device(steps)
        props.append(p)
    for p in props:
        p.synchronize()
    t0 = time.perf_counter()
    for p in props:
        p.run_device(steps)
    for p in props:
        p.synchronize()
    t_plain = time.perf_counter() - t0
    v_p = sum(c["width"] * c["height"] for c, _ in small[:48]) * steps / t_plain
    for p in props:
        p.close()
    out["small_worlds_batched_over_plain"] = {
        "batched": v_b, "plain": v_p, "ratio": v_b / v_p,
        "workload": "1024 worlds with sides {64,96,128} per axis (plain: 48 of them, one propagator each, "
                    "graph-replayed, each on its own stream, enqueued in turn); both timed the same way after a "
                    "warm-up of the same length: host wall time around device-synchronised run(48) calls on the "
                    "public API"}
    return out


def measure_adjoint(args, dist):
    """Differentiable step: `--adjoint-worlds` worlds of 256x256, 2 channels,
    4 kernels (every source->target pair, 1-3 rings, multispecies parameter
    distributions), R=13; forward T steps keeping every k-th state, then the
    reverse sweep for L = sum (A_T - target)^2, target = A_0 shifted 20 cells
    along x.  Device time of each pass from CUDA events on the engine's stream,
    median of 3 after one warm-up pass."""
    import autoverse_b200 as fl
    from autoverse_b200 import workloads as wl
    worlds = wl.adjoint_worlds(args.adjoint_worlds, size=256, R=13, seed=wl.DEFAULT_SEED + RANK)
    b = fl.AdjointBatch([c for c, _ in worlds])
    tgt = []
    for i, (c, sd) in enumerate(worlds):
        a0 = fl.SimulationState.from_seed(sd, c).channels
        b.write_state(i, a0)
        tgt.append(wl.shifted(a0, 256, 256, 20))
    tgt = np.stack(tgt)
    T, k = args.adjoint_steps, args.adjoint_every
    fw, bw = [], []
    for it in range(4):  # pass 0 is the warm-up
        b.forward(T, k)
        fin = np.stack([b.read_final(i) for i in range(b.n_worlds)])
        b.backward(2.0 * (fin - tgt))
        f, g = b.timings()
        if it:
            fw.append(f)
            bw.append(g)
    b.close()
    f = reduce_max(dist, float(np.median(fw)))
    g = reduce_max(dist, float(np.median(bw)))
    cells = args.adjoint_worlds * 256 * 256 * T * WORLD
    return {"workload": f"{args.adjoint_worlds} worlds per GPU of 256x256, C=2, K=4, R=13, T={T}, checkpoint every {k}, "
                        "loss sum (A_T - shift_x(A_0, 20))^2, gradients for A_0, beta_a, weight, mu, sigma and ring "
                        "amplitude/distance/width",
            "forward_ms": f, "backward_ms": g, "backward_over_forward": g / f,
            "forward_cell_steps_per_s": cells / (f / 1e3), "backward_cell_steps_per_s": cells / (g / 1e3)}


def measure_fitness(args, dist):
    """Population fitness: `--fitness-candidates` candidates (worlds of sides
    {64,96,128}, 1-2 channels, the batched-world parameter distributions) each
    evaluated for 200 steps with a sample every 10 and the reference's default
    metrics (Persistence 1.0, Compactness 0.5), all in one batch through the
    public API; wall clock around the whole evaluation.  CPU leg: the
    restatement of the reference's evaluator over the oracle, one candidate
    after another on one core, on the first 4 candidates."""
    import autoverse_b200.fitness as FT
    from autoverse_b200 import workloads as wl
    pop = wl.batched_worlds(args.fitness_candidates, sides=(64, 96, 128), seed=wl.DEFAULT_SEED + 23 + RANK)
    cfgs, seeds = [c for c, _ in pop], [s for _, s in pop]
    # warm-up: 64 candidates cover every size class, so no kernel is first
    # loaded inside the timed evaluation
    FT.evaluate_population(cfgs[:64], seeds[:64], evaluation={"steps": 10})
    t0 = time.perf_counter()
    tm = {}
    res = FT.evaluate_population(cfgs, seeds, timings=tm)
    t = reduce_max(dist, time.perf_counter() - t0)
    cells = sum(c["width"] * c["height"] for c in cfgs)
    out = {"workload": f"{args.fitness_candidates} candidates per GPU, sides {{64,96,128}}, 200 steps, sample every 10, "
                       "metrics Persistence 1.0 + Compactness 0.5",
           "candidates_per_s": WORLD * len(cfgs) / t, "cell_steps_per_s": WORLD * cells * 200 / t, "seconds": t,
           "mean_fitness": float(np.mean([r["fitness"] for r in res])), "seconds_split": tm}
    # the next generation of an evolution run (same layouts, mutated kernel,
    # growth and flow parameters) on the evaluator's batch of the first one
    nxt = wl.mutated_worlds(pop, wl.DEFAULT_SEED + 24 + RANK)
    with FT.PopulationEvaluator() as ev:
        ev.evaluate(cfgs, seeds)
        t0 = time.perf_counter()
        tm2 = {}
        ev.evaluate([c for c, _ in nxt], [s for _, s in nxt], timings=tm2)
        t2 = reduce_max(dist, time.perf_counter() - t0)
        reused = ev.batches_reused
    out["next_generation"] = {"candidates_per_s": WORLD * len(cfgs) / t2, "seconds": t2, "seconds_split": tm2,
                              "batch_reused": bool(reused)}
    if RANK == 0 and not args.skip_cpu:
        import multiprocessing as mp
        from oracle import fitness_ref as FR
        threads = os.cpu_count() or 1
        n = 2 * threads
        work = [(c, sd, FT.DEFAULT_FITNESS, FT.DEFAULT_EVALUATION) for c, sd in zip(cfgs[:n], seeds[:n])]
        # worker processes are spawned (not forked: this process holds a CUDA context)
        with mp.get_context("spawn").Pool(threads) as pool:
            pool.starmap(FR.evaluate, work[:threads])  # warm-up: workers import and load the oracle
            t0 = time.perf_counter()
            pool.starmap(FR.evaluate, work, chunksize=1)
            dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"candidates_per_s": n / dt, "cores": threads, "kind": "port",
                               "sample": f"the first {n} candidates, one per host process on {threads} cores (the "
                                         "reference evaluates candidates in parallel on a rayon pool)"}
    return out


def embedded_workload(side: int):
    """Two species in one 2-channel world: kernels for all 4 channel pairs
    (R = 13, the reference's default kernel radius), the left and right halves
    seeded with distinct CellParams, 20 U(0,1) 24x24 patches per channel,
    softmax mixing at temperature 1."""
    from autoverse_b200 import workloads as wl
    rng = np.random.default_rng(wl.DEFAULT_SEED + 31)
    ks = [wl.kernel(src=i, tgt=j, rings=wl.random_rings(rng), mu=float(rng.uniform(0.12, 0.18)),
                    sigma=float(rng.uniform(0.012, 0.02))) for i in range(2) for j in range(2)]
    cfg = wl.config(side, side, 2, ks, kernel_radius=13)
    cfg["embedding"] = {"enabled": True, "mixing_temperature": 1.0, "linear_mixing": False}
    st = np.zeros((2, side, side), np.float32)
    for c in range(2):
        for _ in range(20):
            x, y = rng.integers(0, side - 24, 2)
            st[c, y:y + 24, x:x + 24] = rng.random((24, 24), dtype=np.float32)
    prm = np.empty((2, side, side, 5), np.float32)
    prm[:, :, : side // 2] = [0.15, 0.015, 1.0, 1.0, 2.0]
    prm[:, :, side // 2:] = [0.2, 0.025, 1.3, 0.8, 2.5]
    return cfg, st.reshape(2, -1), prm.reshape(2, -1, 5)


def measure_embedded(args, dist):
    """Parameter-embedded world (EmbeddedPropagator): device time of 208
    graph-replayed steps after 32 warm-up steps, plus per-kernel times of 20
    eager steps.  CPU leg: the oracle's restatement of the reference's
    single-threaded EmbeddedPropagator::step on 2 steps of the same world."""
    import autoverse_b200 as fl
    side = args.embedded_size
    cfg, st, prm = embedded_workload(side)
    steps = 208
    with fl.EmbeddedPropagator(cfg) as p:
        p.write(fl.EmbeddedState(st, prm, side, side))
        p.run_device(32)
        p.synchronize()
        if dist:
            dist.barrier()
        ms = reduce_max(dist, p.profile_run(steps)["step_ms"])
        stages = p.profile_run(20, stages=True)["stages"]
        p.synchronize()
    cells = side * side
    out = {"workload": f"{side}x{side} torus, 2 channels, 4 kernels (all pairs), R=13, two species (left/right "
                       "CellParams), 20 U(0,1) 24x24 patches per channel, softmax mixing T=1",
           "steps": steps, "us_per_step": 1e3 * ms / steps, "cell_steps_per_s": WORLD * cells * steps / (ms * 1e-3),
           "stage_us_per_step": {k: 1e3 * v / 20 for k, v in stages.items()}}
    if RANK == 0 and not args.skip_cpu:
        from oracle import oracle as O
        o = O.OracleEmbedded(cfg)
        o.run(st, prm, 1)
        t0 = time.perf_counter()
        o.run(st, prm, 2)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"cell_steps_per_s": cells * 2 / dt, "cores": 1, "kind": "port",
                               "sample": "2 steps of the same world, C restatement of EmbeddedPropagator::step "
                                         "(single-threaded, as the reference's)"}
    return out


def measure_recording(args, dist, cfg, state, mode):
    """Animation recording of the headline world: `--record-steps` single
    steps with a frame every 10 steps written to an FLWA file in the system's
    temporary directory (wall clock including the finalize that waits for the
    last frame), against the same single steps without recording."""
    import autoverse_b200 as fl
    n = args.record_steps
    with fl.CudaPropagator(cfg, conv_mode=mode) as p:
        p.write_state(state)
        for _ in range(16):
            p.run_device(1)
        p.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            p.run_device(1)
        p.synchronize()
        plain = time.perf_counter() - t0
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "bench.flwa")
            rec = fl.AnimationRecorder(path, p, frame_skip=10)
            t0 = time.perf_counter()
            rec.run(n)
            stats = rec.finalize()
            t = time.perf_counter() - t0
    t, plain = reduce_max(dist, t), reduce_max(dist, plain)
    return {"workload": f"{n} single steps of the headline world, a frame every 10 steps "
                        f"({stats['frame_count']} frames of {stats['average_frame_size'] / 2**20:.1f} MiB)",
            "steps_per_s_recording": n / t, "steps_per_s_without": n / plain, "overhead": t / plain - 1.0,
            "frames": stats["frame_count"], "mib_per_s_written": stats["total_bytes"] / 2**20 / t}


def measure_other_configs(args, dist, headline: str):
    """The other single-world configurations on the same path (blob 256^2,
    1 channel, R=13; sphere 128^3, R=10): device step rate with the L2 flushed
    before every step, the per-kernel split and the dominant kernel's fraction
    of the measured HBM bandwidth."""
    import autoverse_b200 as fl
    peak, _ = hbm_peak()
    out = {}
    for name in ("blob256", "sphere128"):
        if name == headline:
            continue
        cfg, state, desc = workload(name, engine=True)
        cells = cfg["width"] * cfg["height"] * cfg.get("depth", 1)
        with fl.CudaPropagator(cfg) as p:
            p.write_state(state)
            p.profile_run(5, flush_l2=True)
            prof = p.profile_run(args.other_steps, flush_l2=True, stages=False)
            t = reduce_max(dist, prof["step_ms"] / 1e3)
            n_st = min(args.other_steps, 300)
            st = p.profile_run(n_st, flush_l2=True, stages=True)["stages"]
            dom = max(st, key=st.get)
            dom_ms = st[dom] / n_st
            b = stage_bytes(cfg, dom)
            ach = b / (dom_ms * 1e-3) / 1e9 if b else None
            out[name] = {"workload": desc["workload"], "conv_path": {fl.CONV_DIRECT: "direct",
                                                                     fl.CONV_FFT: "fft"}[p.conv_mode],
                         "steps": args.other_steps, "us_per_step": 1e6 * t / args.other_steps,
                         "value": WORLD * cells * args.other_steps / t, "unit": "cell-steps/s",
                         "stage_us_per_step": {k: 1e3 * v / n_st for k, v in st.items()},
                         "roofline": {"kernel": dom, "achieved": ach, "unit": "GB/s",
                                      "frac": ach / peak if ach else None, "algorithmic_bytes_per_launch": b},
                         "l2": "flushed before every timed step"}
    return out


def measure_sweep(args, dist):
    """Parameter sweep: `--sweep-worlds` worlds of 256x256, 2 channels, 4
    kernels with one set of kernel shapes and per-world weights, mu, sigma,
    dt and beta_a, so the batch keeps one kernel-spectrum set; the same sweep
    with a ring draw per world (the same per-step work, a spectrum set per
    world) beside it.  Device time of 48 graph-replayed steps after 16, and
    the host time of creating the batch."""
    import autoverse_b200 as fl
    from autoverse_b200 import workloads as wl
    out = {"workload": f"{args.sweep_worlds} worlds per GPU of 256x256, C=2, K=4, R=13, per-world weight/mu/sigma/"
                       "dt/beta_a, Gaussian blobs"}
    for name, distinct in (("shared_kernels", False), ("distinct_kernels", True)):
        worlds = wl.sweep_worlds(args.sweep_worlds, seed=wl.DEFAULT_SEED + 41 + RANK, distinct_kernels=distinct)
        t0 = time.perf_counter()
        b = fl.BatchedPropagator([c for c, _ in worlds])
        setup = time.perf_counter() - t0
        for i, (_, sd) in enumerate(worlds):
            b.load_seed(i, sd)
        b.run(16)
        b.synchronize()
        if dist:
            dist.barrier()
        ms = reduce_max(dist, b.profile_run(48, flush_l2=False, stages=False)["step_ms"])
        info = b.info()
        out[name] = {"ms_per_step": ms / 48, "cell_steps_per_s": WORLD * info["cells"] * 48 / (ms * 1e-3),
                     "create_s": setup, "kernel_spectra": info["kernel_spectra"],
                     "kernel_spectra_mib": info["kernel_spectra_bytes"] / 2**20}
        b.close()
    return out


def main():
    args = parse_args()
    cfg, state, desc = workload(args.workload, engine=args.impl == "engine")
    W, H, C = cfg["width"], cfg["height"], cfg["channels"]
    cells = W * H * cfg.get("depth", 1)
    metric = "cell-steps/s on 1 B200, batched vs plain at \u22641e-5 err; backward/forward ratio"

    if args.impl == "reference":
        dist = dist_init()
        if RANK != 0:
            return
        budget = 60.0
        warm = max(3, min(args.warmup, 10))  # at least 3 untimed steps; a CPU step takes about 0.1 s
        n, dt, threads = cpu_reference_run(cfg, state, budget, max(args.steps, 1), warmup=warm)
        v = cells * n / dt
        line = {"metric": metric, "value": v, "unit": "cell-steps/s", "n_gpus": args.gpus, "steps": n,
                "warmup": warm, "ms_per_step": 1e3 * dt / n, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, 0x5EED)",
                "config": dict(desc, parallelism="host threads"), "impl": "reference",
                "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": threads, "kind": "port",
                                 "sample": f"{n} of {args.steps} requested steps (time-bounded at {budget:.0f} s) "
                                           "of the same workload; C restatement of CpuPropagator, f32"},
                "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import autoverse_b200 as fl
    from autoverse_b200 import _native as nat
    dist = dist_init()
    dev = nat.device_info()
    p = fl.CudaPropagator(cfg, conv_mode={"auto": fl.CONV_AUTO, "direct": fl.CONV_DIRECT,
                                          "fft": fl.CONV_FFT}[args.conv])
    if args.tuning:
        v = [int(x) for x in args.tuning.split(",")]
        p.set_tuning(conv_mode=p.conv_mode, wpc_r2c=v[0], wpc_cols=v[1], share_cols=v[2], wpc_c2r=v[3], gather_gby=v[4])
    mode = {fl.CONV_DIRECT: "direct", fl.CONV_FFT: "fft"}[p.conv_mode]
    tuning = p.tuning()
    p.write_state(state)
    flush = not args.no_flush
    # warm-up (untimed)
    p.profile_run(max(args.warmup, 3), flush_l2=flush)
    if dist:
        dist.barrier()
    sampler = ClockSampler(dev["pci_bus_id"]) if RANK == 0 else None
    if sampler:
        sampler.start()
    # the timed K steps: one event pair per step, no events between kernels
    prof = p.profile_run(args.steps, flush_l2=flush, stages=False)
    clocks = sampler.stop() if sampler else None
    p.synchronize()
    t_local = prof["step_ms"] / 1e3
    t = reduce_max(dist, t_local)
    value = WORLD * cells * args.steps / t
    # per-kernel breakdown in a second pass with events around every kernel
    stage_steps = min(args.steps, 1000)
    sprof = p.profile_run(stage_steps, flush_l2=flush, stages=True)
    stages = sprof["stages"]
    dom = max(stages, key=stages.get)
    dom_ms = stages[dom] / stage_steps
    dom_bytes = stage_bytes(cfg, dom)
    peak, peak_kind = hbm_peak()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9 if dom_bytes else None
    traffic = None
    prof_json = os.path.join(ROOT, "profiles", f"{dom}_{args.workload}.json")
    if os.path.exists(prof_json):
        with open(prof_json) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")

    # end to end through the public API on a state in pinned host memory, the
    # reference's step(&mut state): every step copies the state in, advances
    # it one step and copies the result back into the same buffer (one C call,
    # one synchronisation)
    pin = fl.propagator.PinnedBuffer(state.shape)
    pin.array[...] = state

    def e2e_step(s):
        p.step_host(pin.array)

    for s in range(4):
        e2e_step(s)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for s in range(args.e2e_steps):
        e2e_step(s)
    e2e_t = reduce_max(dist, time.perf_counter() - t0)
    e2e_value = WORLD * cells * args.e2e_steps / e2e_t
    # the same host-state call advancing 10 steps per call (run(&mut state, 10))
    calls = max(1, args.e2e_steps // 10)
    p.step_host(pin.array, steps=10)
    t0 = time.perf_counter()
    for _ in range(calls):
        p.step_host(pin.array, steps=10)
    e2e10_t = reduce_max(dist, time.perf_counter() - t0)
    e2e10_value = WORLD * cells * 10 * calls / e2e10_t

    batched = measure_batched(args, dist) if args.batch_worlds > 0 else None
    adjoint = measure_adjoint(args, dist) if args.adjoint_worlds > 0 else None
    fitness = measure_fitness(args, dist) if args.fitness_candidates > 0 else None
    embedded = measure_embedded(args, dist) if args.embedded_size > 0 else None
    recording = measure_recording(args, dist, cfg, state, p.conv_mode) if args.record_steps > 0 else None
    sweep = measure_sweep(args, dist) if args.sweep_worlds > 0 else None
    others = measure_other_configs(args, dist, args.workload) if args.other_steps > 0 else None

    cpu = None
    if RANK == 0 and WORLD == 1 and not args.skip_cpu:
        n, dt, threads = cpu_reference_run(cfg, state, args.cpu_seconds, 200)
        cpu = {"value": cells * n / dt, "unit": "cell-steps/s", "cores": threads, "kind": "port",
               "sample": f"{n} steps of the same workload (time-bounded at {args.cpu_seconds:.0f} s, 1 warm-up), "
                         "C restatement of CpuPropagator in f32, OpenMP over kernels/channels"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if RANK != 0:
        return
    line = {
        "metric": metric, "value": value, "unit": "cell-steps/s", "n_gpus": WORLD, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, 0x5EED)",
        "config": dict(desc, conv_path=mode, launch_choices={k: tuning[k] for k in p.TUNING_FIELDS[1:]}, parallelism=("replicas x%d" % WORLD) if WORLD > 1 else "single GPU",
                       l2="flushed before every timed step" if flush else "warm"),
        "cell_channel_steps_per_s": value * C,
        "stage_ms_per_step": {k: v / stage_steps for k, v in stages.items()},
        "stage_breakdown": f"{stage_steps} further steps with CUDA events around every kernel",
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback 6.65 TB/s", "algorithmic_bytes_per_launch": dom_bytes},
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": int(state.nbytes),
                "d2h_bytes_per_step": int(state.nbytes), "steps": args.e2e_steps},
        "e2e_10_steps_per_call": {"value": e2e10_value, "unit": "cell-steps/s", "calls": calls,
                                  "h2d_bytes_per_call": int(state.nbytes), "d2h_bytes_per_call": int(state.nbytes)},
        "gpu_launches": prof["launches_per_step"] * args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "batched": batched,
        "batched_over_plain": batched["small_worlds_batched_over_plain"]["ratio"] if batched else None,
        "adjoint": adjoint,
        "backward_over_forward": adjoint["backward_over_forward"] if adjoint else None,
        "fitness": fitness,
        "embedded": embedded,
        "recording": recording,
        "sweep": sweep,
        "other_configs": others,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
