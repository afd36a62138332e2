"""The FP64 taped reference gradient (oracle/adjoint_ref.py) pinned against
the FP64 oracle: its forward reproduces the oracle's T steps, and its
gradients match fourth-order central finite differences of the oracle's
loss in every parameter and in sampled state entries."""
import numpy as np
import pytest

from autoverse_b200 import workloads as wl
from oracle import adjoint_ref as AR
from oracle import oracle as O

T = 3


@pytest.fixture(scope="module")
def case():
    (cfg, sd), = wl.adjoint_worlds(1, size=48, R=8, seed=7)
    st = O.seed_generate(sd, cfg)
    tgt = wl.shifted(st, 48, 48, 4)
    L, AT, gA, gp = AR.loss_and_grads(cfg, st, tgt, T)
    return cfg, st, tgt, L, AT, gA, gp


def test_taped_forward_matches_fp64_oracle(case):
    cfg, st, tgt, L, AT, *_ = case
    exp = O.OraclePropagator(cfg, f64=True, exact_params=True).run(st.astype(np.float64), T)
    assert np.abs(AT - exp).max() < 1e-12
    assert L == pytest.approx(float(((exp - tgt) ** 2).sum()), rel=1e-12)


def test_param_layout_round_trip(case):
    cfg = case[0]
    p = AR.param_vector(cfg)
    assert len(p) == len(AR.param_names(cfg)) == 1 + sum(3 + 3 * len(k["rings"]) for k in cfg["kernels"])
    assert AR.param_vector(AR.with_params(cfg, p)) == p


def test_taped_param_grads_match_finite_differences(case):
    cfg, st, tgt, L, AT, gA, gp = case
    scale = np.abs(gp).max()
    for i in range(len(gp)):
        fd = AR.fd_param_grad(cfg, st, tgt, T, i)
        assert abs(gp[i] - fd) <= 1e-6 * max(abs(fd), 1e-3 * scale), (AR.param_names(cfg)[i], gp[i], fd)


def test_taped_state_grads_match_finite_differences(case):
    cfg, st, tgt, L, AT, gA, gp = case
    g = gA.reshape(-1)
    rng = np.random.default_rng(1)
    big = np.flatnonzero(np.abs(g) > 1e-2 * np.abs(g).max())
    for idx in rng.choice(big, 6, replace=False):
        fd = AR.fd_state_grad(cfg, st, tgt, T, int(idx))
        assert abs(g[idx] - fd) <= 1e-6 * abs(fd), (idx, g[idx], fd)
