"""FP64 taped reference gradient of T Flow Lenia steps — TEST INFRASTRUCTURE ONLY.

A differentiable restatement of the reference's 2D step (CpuPropagator::step,
src/compute/propagator.rs:239-420) in float64 torch tensors, so that autograd
records the tape and replays it backwards.  Only the test suite uses it, as
the checker of the engine's hand-written adjoint; the engine never calls it.

Pieces, each following the reference file it cites:
  * kernel      kernel.rs:32-92   sum of Gaussian rings over the normalised
                                  distance, masked at 1, normalised to sum 1;
                kernel.rs:98-117  wrap-padding with the centre at [0, 0]
  * conv        fft.rs:288-324    circular convolution (here torch.fft, f64)
  * growth      growth.rs:45-59   U_t += w (2 exp(-(u-mu)^2 / (2 sigma^2)) - 1)
  * Sobel       gradient.rs:68-108 3x3 Sobel x 1/8 on the torus
  * alpha/flow  flow.rs:14-32, 68-87
  * advection   reintegration.rs:60-167: each source with |m| >= 1e-10 moves
                to x + dt F and deposits m * overlap / (2s)^2 into the cells
                its square of half-side s overlaps (torus wrap)

Parameter vector of one world (the layout of the engine's adjoint API):
  [beta_a] + for each kernel [weight, mu, sigma] + for each of its rings
  [amplitude, distance, width].
"""
from __future__ import annotations

import math
from typing import Sequence

import numpy as np
import torch

DT = torch.float64


def param_vector(cfg: dict) -> list[float]:
    out = [float(cfg["flow"]["beta_a"])]
    for k in cfg["kernels"]:
        out += [float(k["weight"]), float(k["mu"]), float(k["sigma"])]
        for r in k["rings"]:
            out += [float(r["amplitude"]), float(r["distance"]), float(r["width"])]
    return out


def param_names(cfg: dict) -> list[str]:
    out = ["beta_a"]
    for i, k in enumerate(cfg["kernels"]):
        out += [f"k{i}.weight", f"k{i}.mu", f"k{i}.sigma"]
        for j, _ in enumerate(k["rings"]):
            out += [f"k{i}.r{j}.amplitude", f"k{i}.r{j}.distance", f"k{i}.r{j}.width"]
    return out


def with_params(cfg: dict, p: Sequence[float]) -> dict:
    """A copy of cfg whose parameters are replaced by the vector p."""
    import copy
    c = copy.deepcopy(cfg)
    c["flow"]["beta_a"] = float(p[0])
    i = 1
    for k in c["kernels"]:
        k["weight"], k["mu"], k["sigma"] = float(p[i]), float(p[i + 1]), float(p[i + 2])
        i += 3
        for r in k["rings"]:
            r["amplitude"], r["distance"], r["width"] = float(p[i]), float(p[i + 1]), float(p[i + 2])
            i += 3
    return c


def _kernel_padded(kcfg: dict, ring_params: list, max_radius: int, W: int, H: int) -> torch.Tensor:
    r = int(round(float(kcfg["radius"]) * max_radius))
    size = 2 * r + 1
    ax = torch.arange(size, dtype=DT) - r
    dist = torch.sqrt(ax[None, :] ** 2 + ax[:, None] ** 2)
    nd = dist / r if r > 0 else dist
    inside = (nd <= 1.0).to(DT)
    val = torch.zeros((size, size), dtype=DT)
    for (b, a, w) in ring_params:
        val = val + b * torch.exp(-((nd - a).abs() ** 2) / (2.0 * w * w))
    val = val * inside
    val = val / val.sum()
    pad = torch.zeros((H, W), dtype=DT)
    ys = (torch.arange(size) - r) % H
    xs = (torch.arange(size) - r) % W
    return pad.index_put((ys[:, None].expand(size, size), xs[None, :].expand(size, size)), val)


def _sobel(f: torch.Tensor):
    def at(dy, dx):
        return torch.roll(f, shifts=(-dy, -dx), dims=(-2, -1))  # value at (y+dy, x+dx)
    tl, tc, tr = at(-1, -1), at(-1, 0), at(-1, 1)
    ml, mr = at(0, -1), at(0, 1)
    bl, bc, br = at(1, -1), at(1, 0), at(1, 1)
    gx = (-tl + tr - 2.0 * ml + 2.0 * mr - bl + br) * 0.125
    gy = (-tl - 2.0 * tc - tr + bl + 2.0 * bc + br) * 0.125
    return gx, gy


def _advect(m: torch.Tensor, fx: torch.Tensor, fy: torch.Tensor, dt: float, s: float) -> torch.Tensor:
    H, W = m.shape
    ys, xs = torch.meshgrid(torch.arange(H, dtype=DT), torch.arange(W, dtype=DT), indexing="ij")
    keep = (m.abs() >= 1e-10).to(DT)
    m = m * keep
    dx = xs + dt * fx
    dy = ys + dt * fy
    area_tot = (2.0 * s) * (2.0 * s)
    out = torch.zeros(H * W, dtype=DT)
    x0 = torch.floor(dx - s).detach()
    y0 = torch.floor(dy - s).detach()
    span = int(math.ceil(2.0 * s)) + 1
    for j in range(span + 1):
        iy = y0 + j
        oh = torch.clamp(torch.minimum(iy + 1.0, dy + s) - torch.maximum(iy, dy - s), min=0.0)
        for i in range(span + 1):
            ix = x0 + i
            ow = torch.clamp(torch.minimum(ix + 1.0, dx + s) - torch.maximum(ix, dx - s), min=0.0)
            contrib = m * (ow * oh) / area_tot
            idx = (torch.remainder(iy, H) * W + torch.remainder(ix, W)).long().reshape(-1)
            out = out.index_add(0, idx, contrib.reshape(-1))
    return out.reshape(H, W)


class TapedWorld:
    """One 2D world whose step is differentiable in its state and parameters."""

    def __init__(self, cfg: dict):
        if cfg.get("depth", 1) != 1:
            raise ValueError("the taped reference covers 2D worlds")
        self.cfg = cfg
        self.W, self.H, self.C = cfg["width"], cfg["height"], cfg["channels"]

    def unpack(self, p: torch.Tensor):
        beta = p[0]
        ks = []
        i = 1
        for k in self.cfg["kernels"]:
            w, mu, sg = p[i], p[i + 1], p[i + 2]
            i += 3
            rings = []
            for _ in k["rings"]:
                rings.append((p[i], p[i + 1], p[i + 2]))
                i += 3
            ks.append((w, mu, sg, rings))
        return beta, ks

    def run(self, A0: torch.Tensor, p: torch.Tensor, steps: int) -> torch.Tensor:
        cfg = self.cfg
        beta, ks = self.unpack(p)
        khat = [torch.fft.rfft2(_kernel_padded(kc, rp, cfg["kernel_radius"], self.W, self.H))
                for kc, (_, _, _, rp) in zip(cfg["kernels"], ks)]
        dt = float(cfg["dt"])
        s = float(cfg["flow"]["distribution_size"])
        n = float(cfg["flow"]["n"])
        A = A0.reshape(self.C, self.H, self.W)
        for _ in range(steps):
            U = [torch.zeros((self.H, self.W), dtype=DT) for _ in range(self.C)]
            spec = {}
            for kc, kh, (w, mu, sg, _) in zip(cfg["kernels"], khat, ks):
                src = kc["source_channel"]
                if src not in spec:
                    spec[src] = torch.fft.rfft2(A[src])
                conv = torch.fft.irfft2(spec[src] * kh, s=(self.H, self.W))
                g = 2.0 * torch.exp(-((conv - mu) ** 2) / (2.0 * sg * sg)) - 1.0
                U[kc["target_channel"]] = U[kc["target_channel"]] + w * g
            S = A.sum(0)
            gsx, gsy = _sobel(S)
            ratio = S / beta
            alpha = torch.clamp(ratio ** n if n not in (1.0, 2.0, 3.0, 4.0) else ratio ** int(n), 0.0, 1.0)
            nxt = []
            for c in range(self.C):
                gux, guy = _sobel(U[c])
                fx = (1.0 - alpha) * gux - alpha * gsx
                fy = (1.0 - alpha) * guy - alpha * gsy
                nxt.append(_advect(A[c], fx, fy, dt, s))
            A = torch.stack(nxt)
        return A.reshape(self.C, -1)


def loss_and_grads(cfg: dict, A0: np.ndarray, target: np.ndarray, steps: int):
    """L = sum (A_T - target)^2 in FP64 with its gradients with respect to the
    initial state and the parameter vector: (L, A_T, dL/dA0, dL/dp)."""
    w = TapedWorld(cfg)
    a = torch.tensor(np.asarray(A0, dtype=np.float64), requires_grad=True)
    p = torch.tensor(param_vector(cfg), dtype=DT, requires_grad=True)
    AT = w.run(a, p, steps)
    L = ((AT - torch.tensor(np.asarray(target, dtype=np.float64))) ** 2).sum()
    L.backward()
    return float(L.detach()), AT.detach().numpy(), a.grad.numpy(), p.grad.numpy()


def _loss_fd(cfg: dict, A0: np.ndarray, target: np.ndarray, steps: int) -> float:
    from . import oracle as O
    AT = O.OraclePropagator(cfg, f64=True, exact_params=True).run(np.asarray(A0, dtype=np.float64), steps)
    return float(((AT - target) ** 2).sum())


def _central(f, h: float) -> float:
    """Fourth-order central difference at step h: (-f(2h) + 8 f(h) - 8 f(-h) + f(-2h)) / 12h."""
    return (-f(2 * h) + 8 * f(h) - 8 * f(-h) + f(-2 * h)) / (12.0 * h)


def fd_param_grad(cfg: dict, A0: np.ndarray, target: np.ndarray, steps: int, index: int, h: float = 1e-6) -> float:
    """Central finite difference of L in parameter `index` (step h, fourth
    order), on the FP64 oracle (the C restatement's double twin, parameters
    taken exactly).  The loss is piecewise smooth: a step of 1e-4 in mu or
    sigma moves enough destinations across a cell edge of the overlap areas
    to bias the quotient by up to a few 1e-3, so the default step is 1e-6,
    where FP64 round-off is still below 1e-8 relative."""
    p = param_vector(cfg)

    def f(d):
        q = list(p)
        q[index] += d
        return _loss_fd(with_params(cfg, q), A0, target, steps)
    return _central(f, h)


def fd_state_grad(cfg: dict, A0: np.ndarray, target: np.ndarray, steps: int, flat_index: int, h: float = 1e-6) -> float:
    def f(d):
        a = np.array(A0, dtype=np.float64).reshape(-1)
        a[flat_index] += d
        return _loss_fd(cfg, a.reshape(np.shape(A0)), target, steps)
    return _central(f, h)
