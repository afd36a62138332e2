"""The engine's hand-written adjoint on the GPU, against the FP64 taped
reference gradient (oracle/adjoint_ref.py, itself pinned to finite
differences of the FP64 oracle) and against finite differences directly.

Loss: L = sum over worlds, channels and cells of (A_T - target)^2 with the
target the initial state shifted along x.  Tolerances: 1e-3 relative (state
gradient in the 2-norm; each parameter against max(|ref|, 1e-2 max|ref|))."""
import numpy as np
import pytest

import autoverse_b200 as fl
from autoverse_b200 import workloads as wl
from oracle import adjoint_ref as AR
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL = 1e-3


def f32_params(cfg):
    return AR.with_params(cfg, [float(np.float32(v)) for v in AR.param_vector(cfg)])


def setup(n=2, size=64, R=9, seed=11, shift=5):
    worlds = wl.adjoint_worlds(n, size=size, R=R, seed=seed)
    cfgs = [f32_params(c) for c, _ in worlds]
    states = [O.seed_generate(sd, c) for c, (_, sd) in zip(cfgs, worlds)]
    targets = [wl.shifted(s, size, size, shift) for s in states]
    return cfgs, states, targets


def run_gpu(cfgs, states, targets, T, k):
    with fl.AdjointBatch(cfgs) as b:
        for i, s in enumerate(states):
            b.write_state(i, s)
        b.forward(T, k)
        fin = np.stack([b.read_final(i) for i in range(len(cfgs))])
        g = 2.0 * (fin - np.stack(targets))
        gA, gp = b.backward(g)
        return fin, gA, gp


def test_forward_is_the_single_world_trajectory():
    cfgs, states, _ = setup(3, seed=12)
    with fl.AdjointBatch(cfgs) as b:
        for i, s in enumerate(states):
            b.write_state(i, s)
        b.forward(10, 4)
        for i, (c, s) in enumerate(zip(cfgs, states)):
            with fl.CudaPropagator(c, conv_mode=fl.CONV_FFT) as p:
                p.write_state(s)
                p.run_device(10)
                assert np.array_equal(b.read_final(i), p.read_state()), i


@pytest.fixture(scope="module")
def grads():
    cfgs, states, targets = setup()
    T, k = 6, 4
    fin, gA, gp = run_gpu(cfgs, states, targets, T, k)
    ref = [AR.loss_and_grads(c, s, t, T) for c, s, t in zip(cfgs, states, targets)]
    return cfgs, states, targets, T, fin, gA, gp, ref


def test_state_gradient_matches_taped_fp64(grads):
    cfgs, states, targets, T, fin, gA, gp, ref = grads
    for i, (L, AT, rA, rp) in enumerate(ref):
        assert np.abs(fin[i] - AT).max() < 1e-4
        err = np.linalg.norm(gA[i].reshape(-1) - rA.reshape(-1)) / np.linalg.norm(rA)
        assert err < REL, (i, err)


def test_param_gradients_match_taped_fp64(grads):
    cfgs, states, targets, T, fin, gA, gp, ref = grads
    for i, (L, AT, rA, rp) in enumerate(ref):
        names = AR.param_names(cfgs[i])
        floor = 1e-2 * np.abs(rp).max()
        for j, n in enumerate(names):
            assert abs(gp[i][j] - rp[j]) <= REL * max(abs(rp[j]), floor), (i, n, gp[i][j], rp[j])


def test_gradients_match_finite_differences(grads):
    cfgs, states, targets, T, fin, gA, gp, ref = grads
    rng = np.random.default_rng(5)
    i = 0
    names = AR.param_names(cfgs[i])
    floor = 1e-2 * np.abs(ref[i][3]).max()
    for j in rng.choice(len(names), 8, replace=False):
        fd = AR.fd_param_grad(cfgs[i], states[i], targets[i], T, int(j))
        assert abs(gp[i][j] - fd) <= REL * max(abs(fd), floor), (names[j], gp[i][j], fd)
    g = gA[i].reshape(-1)
    big = np.flatnonzero(np.abs(g) > 0.05 * np.abs(g).max())
    for idx in rng.choice(big, 4, replace=False):
        fd = AR.fd_state_grad(cfgs[i], states[i], targets[i], T, int(idx))
        assert abs(g[idx] - fd) <= REL * abs(fd) + 1e-4 * np.abs(g).max(), (idx, g[idx], fd)


def test_checkpoint_interval_does_not_change_gradients():
    cfgs, states, targets = setup(2, seed=13)
    _, gA1, gp1 = run_gpu(cfgs, states, targets, 5, 1)
    _, gA5, gp5 = run_gpu(cfgs, states, targets, 5, 5)
    _, gA2, gp2 = run_gpu(cfgs, states, targets, 5, 2)
    assert np.array_equal(gA1, gA5) and np.array_equal(gA1, gA2)
    for a, b, c in zip(gp1, gp5, gp2):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(a, c, rtol=1e-9, atol=1e-12)


def test_adjoint_errors():
    cfgs, states, targets = setup(2, seed=14)
    other = f32_params(wl.adjoint_worlds(1, size=96, R=9, seed=1)[0][0])
    with pytest.raises(fl.FlpError):
        fl.AdjointBatch([cfgs[0], other])
    with fl.AdjointBatch(cfgs) as b:
        with pytest.raises(fl.FlpError):
            b.backward(np.zeros((2, b.C, b.H * b.W), np.float32))
        with pytest.raises(fl.FlpError):
            b.forward(0, 4)
