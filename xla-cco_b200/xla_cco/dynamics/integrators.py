"""MD integrators: velocity Verlet, Andersen resets, Langevin BAOAB.

Same functions and step arithmetic as ``xla_cco/dynamics/integrators.py``
of the reference (mass 1, Cartesian arrays):

* ``verlet_step``: v += dt/2 F; r += dt v; F = F(r); v += dt/2 F.
* ``andersen_reset``: "count" (acc += p; if acc >= 1 one uniformly chosen
  particle's velocity is redrawn from N(0, T) and acc -= 1) or "bernoulli"
  (one redraw with probability p).
* ``baoab_step``: B, A, O (v = c v + sqrt((1 - c^2) T) xi, c = exp(-gamma
  dt)), A, force, B.

These single steps take any ``force_fn`` (r -> (Phi, F, re, im)) and run as
array code on the caller's side (NumPy, or torch on the GPU). ``md_run``
advances a batch of lanes by many steps on the device (``cco_md_run``): one
force evaluation per step, the step arithmetic fused into the tick, the
force from the stealthy kernels.

Random draws. The reference splits JAX threefry keys; here a key is a pair
of uint32 and every draw is Philox4x32-10 (Salmon et al., SC11) of the key
with the counter (0, 0, stream, index), streams 1 (BAOAB noise, index =
element), 3 (Andersen coin), 4 (particle pick), 5 (velocity row, index =
axis); a step returns the key Philox(key, (0, 0, 7, 0))[:2]. The device uses
the same streams, so ``md_run`` equals these steps chained on their returned
keys. Normals: Box-Muller on two 53-bit uniforms.
"""

from __future__ import annotations

import ctypes
import dataclasses
import math
from typing import Any, Callable, Tuple

import numpy as np

from xla_cco import _native
from xla_cco._types import require_float64

__all__ = [
    "verlet_step", "andersen_reset", "baoab_step", "make_force_fn", "make_key", "MDStepSettings",
    "md_run", "ANDERSEN_MODES",
]  # fmt: skip

ANDERSEN_MODES = ("count", "bernoulli")
ForceFn = Callable[[Any], Tuple[Any, Any, Any, Any]]

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)
_NOISE, _COIN, _PICK, _ROW, _NEXT = 1, 3, 4, 5, 7


def philox4x32_10(key: np.ndarray, counters: np.ndarray) -> np.ndarray:
    """Philox4x32-10 (Salmon et al., SC11) of (len, 4) uint32 counters under a
    uint32[2] key; returns (len, 4) uint32."""
    c = np.array(counters, dtype=np.uint32).reshape(-1, 4)
    k0, k1 = np.uint32(key[0]), np.uint32(key[1])
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = _M0 * c[:, 0].astype(np.uint64)
            p1 = _M1 * c[:, 2].astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & _MASK).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & _MASK).astype(np.uint32)
            c = np.stack([hi1 ^ c[:, 1] ^ k0, lo1, hi0 ^ c[:, 3] ^ k1, lo0], axis=1)
            k0 = np.uint32(k0 + _W0)
            k1 = np.uint32(k1 + _W1)
    return c


def _philox(key: np.ndarray, stream: int, index: Any) -> np.ndarray:
    """Draws of one stream: counters (0, 0, stream, index)."""
    idx = np.asarray(index, dtype=np.uint32).reshape(-1)
    c = np.zeros((idx.size, 4), dtype=np.uint32)
    c[:, 2] = np.uint32(stream)
    c[:, 3] = idx
    return philox4x32_10(key, c)


def _u53(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return ((a.astype(np.uint64) >> np.uint64(5)) << np.uint64(26) |
            (b.astype(np.uint64) >> np.uint64(6))).astype(np.float64) * 2.0**-53  # fmt: skip


def _normal(w: np.ndarray) -> np.ndarray:
    u1 = 1.0 - _u53(w[:, 0], w[:, 1])
    u2 = _u53(w[:, 2], w[:, 3])
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def make_key(seed: int) -> np.ndarray:
    """A key (uint32[2]) from an integer seed."""
    s = int(seed) & 0xFFFFFFFFFFFFFFFF
    return np.array([s & 0xFFFFFFFF, s >> 32], dtype=np.uint32)


def _next_key(key: np.ndarray) -> np.ndarray:
    return _philox(key, _NEXT, [0])[0, :2].copy()


def _check_phase_space(r: Any, v: Any, f: Any, dt: float) -> None:
    for x, name in ((r, "r"), (v, "v"), (f, "f")):
        require_float64(x, name)
    if r.ndim != 2 or tuple(v.shape) != tuple(r.shape) or tuple(f.shape) != tuple(r.shape):
        raise ValueError(f"r, v, f must share an (n, d) shape: {tuple(r.shape)}, "
                         f"{tuple(v.shape)}, {tuple(f.shape)}")  # fmt: skip
    if not (math.isfinite(dt) and dt > 0.0):
        raise ValueError(f"dt must be finite and positive, got {dt}")


def _like(x: Any, ref: Any) -> Any:
    """``x`` (NumPy) as the array type of ``ref``."""
    if hasattr(ref, "device") and hasattr(ref, "dtype") and not isinstance(ref, np.ndarray):
        import torch

        return torch.as_tensor(x, dtype=torch.float64, device=ref.device)
    return x


def verlet_step(r: Any, v: Any, f: Any, force_fn: ForceFn, dt: float):
    """One velocity-Verlet step; returns (r', v', force_fn(r'))."""
    _check_phase_space(r, v, f, dt)
    half = 0.5 * dt
    v_half = v + half * f
    r_new = r + dt * v_half
    out = force_fn(r_new)
    assert len(out) == 4, "force_fn must return (Phi, F, re, im)"
    return r_new, v_half + half * out[1], out


def andersen_reset(key: np.ndarray, v: Any, reset_acc: float, temperature: float, p: float,
                   mode: str):  # fmt: skip
    """Andersen resets after a step; returns (key', v', reset_acc', n_reset)."""
    if mode not in ANDERSEN_MODES:
        raise ValueError(f"mode must be one of {ANDERSEN_MODES}, got {mode!r}")
    if not 0.0 <= p <= 1.0:
        raise ValueError(f"p must lie in [0, 1], got {p}")
    require_float64(v, "v")
    if v.ndim != 2:
        raise ValueError(f"v must have shape (n, d), got {tuple(v.shape)}")
    n, d = v.shape
    if mode == "count":
        acc = float(reset_acc) + p
        fire = acc >= 1.0
        acc = acc - 1.0 if fire else acc
    else:
        w = _philox(key, _COIN, [0])[0]
        fire = bool(_u53(w[:1], w[1:2])[0] < p)
        acc = float(reset_acc)
    q = _philox(key, _PICK, [0])[0]
    pick = min(int(_u53(q[:1], q[1:2])[0] * n), n - 1)
    v_new = v
    if fire:
        row = math.sqrt(float(temperature)) * _normal(_philox(key, _ROW, np.arange(d)))
        v_new = v.clone() if hasattr(v, "clone") else v.copy()
        v_new[pick] = _like(row, v)
    return _next_key(key), v_new, acc, int(fire)


def baoab_step(key: np.ndarray, r: Any, v: Any, f: Any, force_fn: ForceFn, dt: float,
               gamma: float, temperature: float):  # fmt: skip
    """One BAOAB Langevin step; returns (key', r', v', force_fn(r'))."""
    _check_phase_space(r, v, f, dt)
    if not (math.isfinite(gamma) and gamma >= 0.0):
        raise ValueError(f"gamma must be finite and >= 0, got {gamma}")
    c = math.exp(-gamma * dt)
    noise = math.sqrt(-math.expm1(-2.0 * gamma * dt) * float(temperature))
    half = 0.5 * dt
    xi = _normal(_philox(key, _NOISE, np.arange(int(np.prod(tuple(r.shape)))))).reshape(tuple(r.shape))
    v = v + half * f
    r = r + half * v
    v = c * v + noise * _like(xi, v)
    r = r + half * v
    out = force_fn(r)
    return _next_key(key), r, v + half * out[1], out


def make_force_fn(energy: Any, basis: Any) -> ForceFn:
    """r -> (Phi, F, re, im) with F = -dPhi/ds B^-T at s = r B^-1 (run.py:219-244)."""
    b = np.asarray(basis, dtype=np.float64)
    d = int(energy.dim)
    if b.shape != (d, d):
        raise ValueError(f"basis must have shape ({d}, {d}), got {b.shape}")
    inv = np.linalg.inv(b)

    def force_fn(r):
        host = isinstance(r, np.ndarray)
        if host:
            s = r @ inv
        else:
            import torch

            s = r @ torch.as_tensor(inv, device=r.device)
        phi, g, re, im = energy.evaluate(s[None], want_rho=True)
        g = g[0]
        f = -(g @ (inv.T if host else torch.as_tensor(inv.T, device=r.device)))
        return phi[0], f, re[0], im[0]

    return force_fn


# ------------------------------------------------------------------ device runs
@dataclasses.dataclass(frozen=True)
class MDStepSettings:
    """Steps of ``md_run``: ``scheme`` "verlet" (optionally with Andersen
    resets) or "baoab"; ``drift_tol`` > 0 stops a lane with STATUS_DRIFT once
    |E - E0| exceeds it."""

    dt: float
    n_steps: int
    scheme: str = "verlet"
    andersen: str = "off"
    andersen_p: float = 0.0
    gamma: float = 0.0
    temperature: float = 0.0
    drift_tol: float = 0.0


def md_run(energy: Any, r0: Any, v0: Any, basis: Any, settings: MDStepSettings, keys: Any,
           reset_acc: Any = None) -> dict:  # fmt: skip
    """Advance (b, n, d) lanes by ``settings.n_steps`` on the device.

    ``keys``: (b, 2) uint32 (or one key for every lane). Returns a dict with
    r, v, f (like r0), and per lane energy, kinetic, max_drift, n_resets,
    reset_acc, keys (the keys of the next step) and status; NumPy in, NumPy
    out, CUDA tensors stay on the device.
    """
    import torch

    if settings.scheme not in ("verlet", "baoab"):
        raise ValueError(f"unknown scheme {settings.scheme!r}")
    if settings.andersen not in ("off",) + ANDERSEN_MODES:
        raise ValueError(f"unknown Andersen mode {settings.andersen!r}")
    require_float64(r0, "r0")
    require_float64(v0, "v0")
    _native.require_gpu()
    host = not (isinstance(r0, torch.Tensor) and r0.is_cuda)
    to_dev = lambda x: (x.detach().to("cuda", torch.float64).contiguous()  # noqa: E731
                        if isinstance(x, torch.Tensor)
                        else torch.from_numpy(np.ascontiguousarray(np.asarray(x))).cuda())  # fmt: skip
    r, v = to_dev(r0), to_dev(v0)
    if r.ndim == 2:
        raise ValueError("md_run takes a (b, n, d) batch")
    b, n, d = r.shape
    dev = r.device
    h = energy.problem_handle(dev.index if dev.index is not None else torch.cuda.current_device(), n)
    handles = (ctypes.c_void_p * b)(*([h] * b))
    bases = np.ascontiguousarray(np.broadcast_to(np.asarray(basis, dtype=np.float64), (b, d, d)))
    k = np.ascontiguousarray(np.broadcast_to(np.asarray(keys, dtype=np.uint32), (b, 2)))
    acc = None if reset_acc is None else np.ascontiguousarray(
        np.broadcast_to(np.asarray(reset_acc, dtype=np.float64), (b,)))  # fmt: skip
    f64, i64 = torch.float64, torch.int64
    out = {"r": torch.empty_like(r), "v": torch.empty_like(r), "f": torch.empty_like(r)}
    for key in ("energy", "kinetic", "max_drift", "reset_acc"):
        out[key] = torch.empty(b, dtype=f64, device=dev)
    out["n_resets"] = torch.empty(b, dtype=i64, device=dev)
    out["status"] = torch.empty(b, dtype=i64, device=dev)
    out["keys"] = torch.empty((b, 2), dtype=torch.int32, device=dev)
    co = _native.MdOutC()
    for key, t in out.items():
        setattr(co, key, t.data_ptr())
    cs = _native.MdSettingsC(
        float(settings.dt), int(settings.n_steps), 1 if settings.scheme == "baoab" else 0,
        {"off": 0, "count": 1, "bernoulli": 2}[settings.andersen], float(settings.andersen_p),
        float(settings.gamma), float(settings.temperature), float(settings.drift_tol),
    )  # fmt: skip
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        code = _native.load().cco_md_run(
            handles, stream, b, r.data_ptr(), v.data_ptr(), bases.ctypes.data, k.ctypes.data,
            acc.ctypes.data if acc is not None else None, ctypes.byref(cs), ctypes.byref(co),
        )  # fmt: skip
    _native.check(code, "cco_md_run")
    res = {key: (t.cpu().numpy() if host else t) for key, t in out.items()}
    kk = out["keys"].cpu().numpy().view(np.uint32)
    res["keys"] = kk if host else out["keys"]
    return res
