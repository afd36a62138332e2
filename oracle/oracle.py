"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

The oracle is a plain-C restatement of the reference crate's CPU Flow Lenia
step (``CpuPropagator``/``CpuPropagator3D``, src/compute/propagator.rs:239-420
and src/compute/propagator3d.rs:119-308).  Only the test suite, the smoke
check and the benchmark's CPU-baseline leg import this module; it is the
checker, never the product.

Configs and seeds are the reference's JSON schema (src/schema/config.rs:14-111,
src/schema/seed.rs:13-135) given as Python dicts.  Floating-point fields are
rounded to f32 the way serde parses an ``f32`` (parse as f64, then cast).
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Any

import numpy as np

from . import build_oracle

_LIBS: dict[str, C.CDLL] = {}


def _lib(f64: bool, tag: str | None = None) -> C.CDLL:
    tag = tag or ("f64" if f64 else "f32")
    if tag not in _LIBS:
        paths = build_oracle.LIBS
        if not os.path.exists(paths[tag]):
            build_oracle.build()
        lib = C.CDLL(paths[tag])
        _declare(lib, "orc64_" if f64 else "orc32_", C.c_double if f64 else C.c_float)
        _LIBS[tag] = lib
    return _LIBS[tag]


def _declare(lib: C.CDLL, p: str, R) -> None:
    P = C.c_void_p
    I = C.c_int
    Z = C.c_size_t
    sig = {
        "kernel_build": (I, [I, R, I, I, P, P]),
        "kernel_pad": (None, [P, I, I, I, I, I, P]),
        "fft_forward": (None, [P, I, I, I, P, P]),
        "fft_inverse": (None, [P, P, I, I, I, P]),
        "fft_convolve": (None, [P, P, I, I, I, P]),
        "direct_convolve2d": (None, [P, P, I, I, I, P]),
        "growth": (R, [R, R, R]),
        "growth_accumulate": (None, [P, P, Z, R, R, R]),
        "sobel2d": (None, [P, P, P, I, I]),
        "sobel3d": (None, [P, P, P, P, I, I, I]),
        "alpha": (R, [R, R, R]),
        "flow_field": (None, [I, P, P, P, Z, R, R, P]),
        "wrap_coord": (I, [I, I]),
        "advect2d": (None, [P, P, P, P, I, I, R, R]),
        "advect3d": (None, [P, P, P, P, P, I, I, I, R, R]),
        "total_mass": (R, [P, Z]),
        "prop_new": (P, [I, I, I, I, R, I, I, P, P, P, R, R, R]),
        "prop_free": (None, [P]),
        "prop_run": (None, [P, P, I, I]),
        "prop_affinity": (None, [P, P, P]),
        "prop_transport": (None, [P, P, P, P]),
        "prop_last_flow": (None, [P, P]),
        "prop_run_many": (None, [P, P, I, I, I]),
        "seed_apply": (None, [P, I, I, I, I, I, P, I, C.c_uint64]),
        "conv_growth_acc_embedded": (None, [P, P, I, P, P, I, I]),
        "distribution_overlap": (R, [R, R, R, R, R]),
        "mix_softmax": (None, [P, P, I, R, P]),
        "mix_linear": (None, [P, P, I, P]),
        "max_flow_magnitude": (R, [P, P, Z]),
        "advect_params2d": (None, [P, P, P, P, I, R, R, R, I, I, P, P]),
        "emb_new": (P, [I, I, I, R, I, I, P, P, P, R, I, I, R]),
        "emb_free": (None, [P]),
        "emb_next_params": (None, [P, P]),
        "emb_step": (None, [P, P, P, I]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, p + name)
        fn.restype = res
        fn.argtypes = args


def _dt(f64: bool):
    return np.float64 if f64 else np.float32


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def _fn(f64: bool, name: str, tag: str | None = None):
    return getattr(_lib(f64, tag), ("orc64_" if f64 else "orc32_") + name)


def f32(x: Any) -> float:
    """serde's f32: parse as f64, round to nearest f32."""
    return float(np.float32(x))


# ---------------------------------------------------------------------------
# Config (src/schema/config.rs:14-164)
# ---------------------------------------------------------------------------

def normalize_config(cfg: dict | str) -> dict:
    if isinstance(cfg, str):
        cfg = json.loads(cfg)
    out = dict(cfg)
    out.setdefault("depth", 1)
    return out


def validate_config(cfg: dict) -> None:
    """config.rs:136-164; raises ValueError like the reference returns ConfigError."""
    if cfg["width"] == 0 or cfg["height"] == 0 or cfg.get("depth", 1) == 0:
        raise ValueError("InvalidDimensions")
    if cfg["channels"] == 0:
        raise ValueError("InvalidChannels")
    if f32(cfg["dt"]) <= 0.0:
        raise ValueError("InvalidTimeStep")
    if cfg["kernel_radius"] == 0:
        raise ValueError("InvalidKernelRadius")
    for i, k in enumerate(cfg["kernels"]):
        if k["source_channel"] >= cfg["channels"] or k["target_channel"] >= cfg["channels"]:
            raise ValueError(f"InvalidChannelIndex kernel {i}")


def _pack_kernels(cfg: dict, f64: bool, exact: bool = False):
    dt = _dt(f64)
    f32 = float if exact else globals()["f32"]
    ks = cfg["kernels"]
    kp = np.zeros((max(len(ks), 1), 6), dtype=dt)
    rc = np.zeros(max(len(ks), 1), dtype=np.int32)
    rings = []
    for i, k in enumerate(ks):
        kp[i] = [f32(k["radius"]), f32(k["weight"]), f32(k["mu"]), f32(k["sigma"]), k["source_channel"],
                 k["target_channel"]]
        rc[i] = len(k["rings"])
        for r in k["rings"]:
            rings.append([f32(r["amplitude"]), f32(r["distance"]), f32(r["width"])])
    ra = np.array(rings if rings else [[0, 0, 0]], dtype=dt)
    return kp, rc, ra


class OraclePropagator:
    """CpuPropagator / CpuPropagator3D restated in C (f32, or f64 twin)."""

    def __init__(self, cfg: dict | str, f64: bool = False, exact_params: bool = False, mass_skip: bool = True):
        """exact_params (f64 only): take the config's numbers as given instead of
        rounding them to f32 first (finite differences of the FP64 twin).
        mass_skip=False (f64 only): the FP64 twin without the reintegration's
        |m| < 1e-10 skip, to measure the mass that the skip removes."""
        if not mass_skip and not f64:
            raise ValueError("the build without the mass skip is FP64 only")
        self._tag = None if mass_skip else "f64_noskip"
        cfg = normalize_config(cfg)
        validate_config(cfg)
        self.cfg = cfg
        self.f64 = f64
        self.W, self.H, self.D = cfg["width"], cfg["height"], cfg["depth"]
        self.C = cfg["channels"]
        self.N = self.W * self.H * self.D
        self.dims = 3 if self.D > 1 else 2
        exact = bool(exact_params and f64)
        kp, rc, ra = _pack_kernels(cfg, f64, exact)
        self._keep = (kp, rc, ra)
        fl = cfg["flow"]
        num = float if exact else f32
        self._h = _fn(f64, "prop_new", self._tag)(self.W, self.H, self.D, self.C, num(cfg["dt"]), cfg["kernel_radius"],
                                      len(cfg["kernels"]), _ptr(kp), _ptr(rc), _ptr(ra), num(fl["beta_a"]),
                                      num(fl["n"]), num(fl["distribution_size"]))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _fn(self.f64, "prop_free", self._tag)(h)
            self._h = None

    def _state(self, state: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(state, dtype=_dt(self.f64)).reshape(self.C, self.N)
        return s.copy()

    def run(self, state: np.ndarray, steps: int = 1, threads: int = 1) -> np.ndarray:
        s = self._state(state)
        _fn(self.f64, "prop_run", self._tag)(self._h, _ptr(s), int(steps), int(threads))
        return s

    def affinity(self, state: np.ndarray) -> np.ndarray:
        s = self._state(state)
        out = np.zeros_like(s)
        _fn(self.f64, "prop_affinity", self._tag)(self._h, _ptr(s), _ptr(out))
        return out

    def transport(self, state: np.ndarray, aff: np.ndarray) -> np.ndarray:
        s = self._state(state)
        a = self._state(aff)
        out = np.zeros_like(s)
        _fn(self.f64, "prop_transport", self._tag)(self._h, _ptr(s), _ptr(a), _ptr(out))
        return out

    def last_flow(self) -> np.ndarray:
        out = np.zeros((self.C, self.dims, self.N), dtype=_dt(self.f64))
        _fn(self.f64, "prop_last_flow", self._tag)(self._h, _ptr(out))
        return out


def run_many(props: list[OraclePropagator], states: list[np.ndarray], steps: int, threads: int) -> list:
    """Advance many independent worlds, parallel over worlds."""
    f64 = props[0].f64
    arrs = [p._state(s) for p, s in zip(props, states)]
    hp = (C.c_void_p * len(props))(*[p._h for p in props])
    sp = (C.c_void_p * len(props))(*[a.ctypes.data for a in arrs])
    _fn(f64, "prop_run_many")(C.cast(hp, C.c_void_p), C.cast(sp, C.c_void_p), len(props), int(steps), int(threads))
    return arrs


# ---------------------------------------------------------------------------
# Seeds (src/schema/seed.rs:160-304)
# ---------------------------------------------------------------------------

_KIND = {"GaussianBlob": 0, "Ring": 1, "GaussianSphere": 2, "Shell": 3, "Torus3D": 4, "Noise": 5}


def seed_generate(seed: dict | str, cfg: dict | str, f64: bool = False) -> np.ndarray:
    """Seed::generate flattened like SimulationState::from_seed: (C, D*H*W)."""
    if isinstance(seed, str):
        seed = json.loads(seed)
    cfg = normalize_config(cfg)
    W, H, D, Cn = cfg["width"], cfg["height"], cfg["depth"], cfg["channels"]
    grid = np.zeros((Cn, D * H * W), dtype=_dt(f64))
    pat = seed["pattern"]
    t = pat["type"]
    apply = _fn(f64, "seed_apply")

    def call(kind, fl, ch, nseed=0):
        fa = np.array(fl + [0.0] * (8 - len(fl)), dtype=_dt(f64))
        apply(_ptr(grid), W, H, D, Cn, kind, _ptr(fa), ch, nseed)

    def blob(b):
        call(0, [f32(b["center"][0]), f32(b["center"][1]), f32(b["radius"]), f32(b["amplitude"])], b["channel"])

    def sphere(s):
        c = s["center"]
        call(2, [f32(c[0]), f32(c[1]), f32(c[2]), f32(s["radius"]), f32(s["amplitude"])], s["channel"])

    if t == "GaussianBlob":
        blob(pat)
    elif t == "MultiBlob":
        for b in pat["blobs"]:
            blob(b)
    elif t == "Ring":
        c = pat["center"]
        call(1, [f32(c[0]), f32(c[1]), f32(pat["inner_radius"]), f32(pat["outer_radius"]), f32(pat["amplitude"])],
             pat["channel"])
    elif t == "GaussianSphere":
        sphere(pat)
    elif t == "MultiSphere":
        for s in pat["spheres"]:
            sphere(s)
    elif t in ("Shell", "Torus3D"):
        c = pat["center"]
        a, b = ("inner_radius", "outer_radius") if t == "Shell" else ("major_radius", "minor_radius")
        call(_KIND[t], [f32(c[0]), f32(c[1]), f32(c[2]), f32(pat[a]), f32(pat[b]), f32(pat["amplitude"])],
             pat["channel"])
    elif t == "Noise":
        ch = pat.get("channel")
        call(5, [f32(pat["amplitude"])], -1 if ch is None else ch, int(pat["seed"]) & 0xFFFFFFFFFFFFFFFF)
    elif t == "Custom":
        mid = D // 2
        for x, y, c, v in pat["values"]:
            if c < Cn and y < H and x < W:
                grid[c, (mid * H + y) * W + x] = f32(v)
    elif t == "Custom3D":
        for x, y, z, c, v in pat["values"]:
            if c < Cn and z < D and y < H and x < W:
                grid[c, (z * H + y) * W + x] = f32(v)
    else:
        raise ValueError(f"unknown pattern type {t}")
    return grid


# ---------------------------------------------------------------------------
# Stage functions (for the reference's own unit tests)
# ---------------------------------------------------------------------------

def kernel_build(kcfg: dict, max_radius: int, dims: int = 2, f64: bool = False) -> np.ndarray:
    rings = np.array([[f32(r["amplitude"]), f32(r["distance"]), f32(r["width"])] for r in kcfg["rings"]] or
                     [[0, 0, 0]], dtype=_dt(f64))
    fn = _fn(f64, "kernel_build")
    size = fn(dims, f32(kcfg["radius"]), max_radius, len(kcfg["rings"]), _ptr(rings), None)
    out = np.zeros((size,) * dims, dtype=_dt(f64))
    fn(dims, f32(kcfg["radius"]), max_radius, len(kcfg["rings"]), _ptr(rings), _ptr(out))
    return out


def kernel_pad(kern: np.ndarray, W: int, H: int, D: int = 1) -> np.ndarray:
    f64 = kern.dtype == np.float64
    k = np.ascontiguousarray(kern)
    out = np.zeros(W * H * D, dtype=k.dtype)
    _fn(f64, "kernel_pad")(_ptr(k), k.shape[0], k.ndim, W, H, D, _ptr(out))
    return out.reshape((D, H, W) if k.ndim == 3 else (H, W))


def fft_forward(x: np.ndarray) -> np.ndarray:
    f64 = x.dtype == np.float64
    x = np.ascontiguousarray(x)
    D, H, W = (1,) * (3 - x.ndim) + x.shape
    re = np.zeros(x.size, dtype=x.dtype)
    im = np.zeros(x.size, dtype=x.dtype)
    _fn(f64, "fft_forward")(_ptr(x), W, H, D, _ptr(re), _ptr(im))
    return (re + 1j * im.astype(np.complex128)).reshape(x.shape)


def fft_inverse(z: np.ndarray, f64: bool = False) -> np.ndarray:
    dt = _dt(f64)
    re = np.ascontiguousarray(z.real, dtype=dt)
    im = np.ascontiguousarray(z.imag, dtype=dt)
    D, H, W = (1,) * (3 - z.ndim) + z.shape
    out = np.zeros(z.size, dtype=dt)
    _fn(f64, "fft_inverse")(_ptr(re), _ptr(im), W, H, D, _ptr(out))
    return out.reshape(z.shape)


def fft_convolve(x: np.ndarray, kern_padded: np.ndarray) -> np.ndarray:
    f64 = x.dtype == np.float64
    x = np.ascontiguousarray(x)
    k = np.ascontiguousarray(kern_padded, dtype=x.dtype)
    D, H, W = (1,) * (3 - x.ndim) + x.shape
    out = np.zeros(x.size, dtype=x.dtype)
    _fn(f64, "fft_convolve")(_ptr(x), _ptr(k), W, H, D, _ptr(out))
    return out.reshape(x.shape)


def direct_convolve2d(x: np.ndarray, kern: np.ndarray, r: int) -> np.ndarray:
    f64 = x.dtype == np.float64
    x = np.ascontiguousarray(x)
    k = np.ascontiguousarray(kern, dtype=x.dtype)
    H, W = x.shape
    out = np.zeros_like(x)
    _fn(f64, "direct_convolve2d")(_ptr(x), _ptr(k), W, H, r, _ptr(out))
    return out


def growth(u: float, mu: float, sigma: float, f64: bool = False) -> float:
    return _fn(f64, "growth")(u, mu, sigma)


def growth_accumulate(conv: np.ndarray, target: np.ndarray, w: float, mu: float, sigma: float) -> np.ndarray:
    f64 = conv.dtype == np.float64
    c = np.ascontiguousarray(conv)
    t = np.ascontiguousarray(target, dtype=c.dtype).copy()
    _fn(f64, "growth_accumulate")(_ptr(c), _ptr(t), c.size, w, mu, sigma)
    return t


def sobel2d(g: np.ndarray):
    f64 = g.dtype == np.float64
    g = np.ascontiguousarray(g)
    H, W = g.shape
    gx = np.zeros_like(g)
    gy = np.zeros_like(g)
    _fn(f64, "sobel2d")(_ptr(g), _ptr(gx), _ptr(gy), W, H)
    return gx, gy


def sobel3d(g: np.ndarray):
    f64 = g.dtype == np.float64
    g = np.ascontiguousarray(g)
    D, H, W = g.shape
    gx, gy, gz = np.zeros_like(g), np.zeros_like(g), np.zeros_like(g)
    _fn(f64, "sobel3d")(_ptr(g), _ptr(gx), _ptr(gy), _ptr(gz), W, H, D)
    return gx, gy, gz


def alpha(mass: float, beta_a: float, n: float, f64: bool = False) -> float:
    return _fn(f64, "alpha")(mass, beta_a, n)


def flow_field(gu: np.ndarray, ga: np.ndarray, mass_sum: np.ndarray, beta_a: float, n: float) -> np.ndarray:
    """gu, ga: (dims, N); returns (dims, N)."""
    f64 = gu.dtype == np.float64
    gu = np.ascontiguousarray(gu)
    ga = np.ascontiguousarray(ga, dtype=gu.dtype)
    ms = np.ascontiguousarray(mass_sum, dtype=gu.dtype)
    out = np.zeros_like(gu)
    _fn(f64, "flow_field")(gu.shape[0], _ptr(gu), _ptr(ga), _ptr(ms), gu.shape[1], beta_a, n, _ptr(out))
    return out


def wrap_coord(c: int, size: int) -> int:
    return _fn(False, "wrap_coord")(c, size)


def advect2d(cur: np.ndarray, fx: np.ndarray, fy: np.ndarray, dt: float, s: float) -> np.ndarray:
    f64 = cur.dtype == np.float64
    cur = np.ascontiguousarray(cur)
    H, W = cur.shape
    fx = np.ascontiguousarray(fx, dtype=cur.dtype)
    fy = np.ascontiguousarray(fy, dtype=cur.dtype)
    nxt = np.zeros_like(cur)
    _fn(f64, "advect2d")(_ptr(cur), _ptr(fx), _ptr(fy), _ptr(nxt), W, H, dt, s)
    return nxt


def advect3d(cur: np.ndarray, fx, fy, fz, dt: float, s: float) -> np.ndarray:
    f64 = cur.dtype == np.float64
    cur = np.ascontiguousarray(cur)
    D, H, W = cur.shape
    fx, fy, fz = (np.ascontiguousarray(a, dtype=cur.dtype) for a in (fx, fy, fz))
    nxt = np.zeros_like(cur)
    _fn(f64, "advect3d")(_ptr(cur), _ptr(fx), _ptr(fy), _ptr(fz), _ptr(nxt), W, H, D, dt, s)
    return nxt


def total_mass(g: np.ndarray) -> float:
    f64 = g.dtype == np.float64
    g = np.ascontiguousarray(g)
    return _fn(f64, "total_mass")(_ptr(g), g.size)


# ---------------------------------------------------------------------------
# EmbeddedPropagator (src/compute/embedded_propagator.rs:222-372,
# direct_convolution.rs:129-177, param_advection.rs:83-165,
# schema/embedding.rs:64-166).  Parameter grids are [channel][cell][5] with the
# fields of CellParams in struct order: mu, sigma, weight, beta_a, n.
# ---------------------------------------------------------------------------

CELL_DEFAULT = (0.15, 0.015, 1.0, 1.0, 2.0)  # CellParams::default (embedding.rs:33-43)
NPAR = 5


def embedding_config(cfg: dict) -> dict:
    """EmbeddingConfig with serde defaults (embedding.rs:331-352)."""
    e = dict(cfg.get("embedding") or {})
    return {"enabled": bool(e.get("enabled", False)), "mixing_temperature": f32(e.get("mixing_temperature", 1.0)),
            "linear_mixing": bool(e.get("linear_mixing", False))}


def default_params(cfg: dict) -> np.ndarray:
    """EmbeddedState::from_seed's parameter grids (embedded_propagator.rs:41-66):
    the first kernel's mu/sigma/weight and the flow's beta_a/n in every cell."""
    ks = cfg["kernels"]
    mu = f32(ks[0]["mu"]) if ks else 0.15
    sigma = f32(ks[0]["sigma"]) if ks else 0.015
    weight = f32(ks[0]["weight"]) if ks else 1.0
    fl = cfg["flow"]
    row = np.array([mu, sigma, weight, f32(fl["beta_a"]), f32(fl["n"])], dtype=np.float32)
    N = cfg["width"] * cfg["height"]
    return np.tile(row, (cfg["channels"], N, 1))


def _rows(params) -> tuple:
    arr = np.ascontiguousarray(np.asarray(params, dtype=np.float32).reshape(-1, NPAR))
    ptrs = (C.c_void_p * len(arr))(*[arr.ctypes.data + i * NPAR * 4 for i in range(len(arr))])
    return arr, ptrs


def mix_softmax(masses, params, temperature: float = 1.0) -> np.ndarray:
    m = np.ascontiguousarray(masses, dtype=np.float32)
    arr, ptrs = _rows(params)
    out = np.zeros(NPAR, dtype=np.float32)
    _fn(False, "mix_softmax")(_ptr(m), C.cast(ptrs, C.c_void_p), len(m), f32(temperature), _ptr(out))
    return out


def mix_linear(masses, params) -> np.ndarray:
    m = np.ascontiguousarray(masses, dtype=np.float32)
    arr, ptrs = _rows(params)
    out = np.zeros(NPAR, dtype=np.float32)
    _fn(False, "mix_linear")(_ptr(m), C.cast(ptrs, C.c_void_p), len(m), _ptr(out))
    return out


def distribution_overlap(dest_x, dest_y, s, cell_x, cell_y) -> float:
    return float(_fn(False, "distribution_overlap")(f32(dest_x), f32(dest_y), f32(s), f32(cell_x), f32(cell_y)))


def conv_growth_embedded(inp: np.ndarray, kern: np.ndarray, params: np.ndarray, W: int, H: int,
                         target: np.ndarray | None = None) -> np.ndarray:
    """convolve_growth_accumulate_embedded into `target` (zeros when None)."""
    x = np.ascontiguousarray(inp, dtype=np.float32).reshape(-1)
    k = np.ascontiguousarray(kern, dtype=np.float32)
    prm = np.ascontiguousarray(params, dtype=np.float32).reshape(-1, NPAR)
    out = np.zeros(W * H, dtype=np.float32) if target is None else np.ascontiguousarray(target, np.float32).copy()
    _fn(False, "conv_growth_acc_embedded")(_ptr(x), _ptr(k), k.shape[0], _ptr(prm), _ptr(out), W, H)
    return out


def advect_params2d(mass, params, fx, fy, W: int, H: int, dt: float, s: float, linear: bool = False,
                    temperature: float = 1.0, next_params: np.ndarray | None = None):
    """advect_mass_and_params_into; returns (next_mass, next_params) with
    next_params starting from `next_params` (CellParams::default grids when None,
    as advect_mass_and_params allocates)."""
    m = np.ascontiguousarray(mass, dtype=np.float32).reshape(-1)
    prm = np.ascontiguousarray(params, dtype=np.float32).reshape(-1, NPAR)
    fxa = np.ascontiguousarray(fx, dtype=np.float32).reshape(-1)
    fya = np.ascontiguousarray(fy, dtype=np.float32).reshape(-1)
    nm = np.zeros(W * H, dtype=np.float32)
    if next_params is None:
        npr = np.tile(np.array(CELL_DEFAULT, dtype=np.float32), (W * H, 1))
    else:
        npr = np.ascontiguousarray(next_params, dtype=np.float32).reshape(-1, NPAR).copy()
    _fn(False, "advect_params2d")(_ptr(m), _ptr(prm), _ptr(fxa), _ptr(fya), int(linear), f32(temperature),
                                  f32(dt), f32(s), W, H, _ptr(nm), _ptr(npr))
    return nm, npr


class OracleEmbedded:
    """EmbeddedPropagator restated in C (f32)."""

    def __init__(self, cfg: dict | str):
        cfg = normalize_config(cfg)
        validate_config(cfg)
        if cfg["depth"] != 1:
            raise ValueError("parameter embedding is 2D only")
        self.cfg = cfg
        self.W, self.H, self.C = cfg["width"], cfg["height"], cfg["channels"]
        self.N = self.W * self.H
        kp, rc, ra = _pack_kernels(cfg, False)
        self._keep = (kp, rc, ra)
        e = embedding_config(cfg)
        self._h = _fn(False, "emb_new")(self.W, self.H, self.C, f32(cfg["dt"]), cfg["kernel_radius"],
                                       len(cfg["kernels"]), _ptr(kp), _ptr(rc), _ptr(ra),
                                       f32(cfg["flow"]["distribution_size"]), int(e["enabled"]),
                                       int(e["linear_mixing"]), e["mixing_temperature"])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _fn(False, "emb_free")(h)
            self._h = None

    def run(self, state: np.ndarray, params: np.ndarray, steps: int = 1):
        """Returns the advanced (state, params); the oracle keeps its own
        parameter buffer across calls, as the reference's propagator does."""
        st = np.ascontiguousarray(state, dtype=np.float32).reshape(self.C, self.N).copy()
        pr = np.ascontiguousarray(params, dtype=np.float32).reshape(self.C, self.N, NPAR).copy()
        _fn(False, "emb_step")(self._h, _ptr(st), _ptr(pr), int(steps))
        return st, pr

    def next_params(self) -> np.ndarray:
        out = np.zeros((self.C, self.N, NPAR), dtype=np.float32)
        _fn(False, "emb_next_params")(self._h, _ptr(out))
        return out
