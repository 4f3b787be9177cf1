"""Gradient flow of the energy landscape (drop-in for ``xla_cco.minimize.flow``).

``gradient_flow(energy, s0, basis, settings, dt0=None)`` integrates the
steepest-descent flow dr/dt = -grad_r Phi in Cartesian coordinates r = s B,
written in fractional coordinates as ds/dt = -grad_s Phi (B B^T)^-1, until a
stop (``minimize/flow.py:258-364`` of the reference). Same settings, stops,
status precedence, clocks (flow time and arclength), recording and result
fields.

* ``method="dopri5"`` runs on the device (``cco_gradient_flow``): each lane
  is a Dormand-Prince 5(4) stage machine advancing one stage evaluation per
  tick; ``s0`` may be (n, d) or a (B, n, d) batch (the reference's vmap).
* ``method="rosenbrock"`` (ROS2 with the exact Hessian, ``flow.py:367-398``)
  is a host-driven loop on the GPU: the closed-form Hessian by DGEMM, an LU
  factorisation and two solves per step (one lane at a time).
"""

from __future__ import annotations

import dataclasses
import math
from typing import Any, Optional

import numpy as np

from xla_cco import _native
from xla_cco._types import require_float64
from xla_cco.minimize.result import (
    STATUS_BUDGET,
    STATUS_ENERGY_TOL,
    STATUS_GRAD_TOL,
    STATUS_RUNNING,
    STATUS_STEP_FLOOR,
)

__all__ = ["FlowSettings", "FlowResult", "FlowTrajectory", "gradient_flow"]

_SAFETY, _SHRINK_MIN, _GROW_MAX = 0.9, 0.2, 5.0
_ROS_GAMMA = 1.0 + 1.0 / math.sqrt(2.0)


@dataclasses.dataclass(frozen=True)
class FlowSettings:
    """Integration controls (same names and defaults as the reference)."""

    rtol: float = 1e-6
    atol: float = 1e-14
    parametrization: str = "time"
    method: str = "dopri5"
    dt_init: float = 1e-3
    dt_min: float = 1e-14
    dt_max: float = math.inf
    t_max: float = math.inf
    max_steps: int = 200_000
    energy_tol: float = 0.0
    grad_tol: float = 0.0
    record_every: int = 0
    max_records: int = 0


@dataclasses.dataclass
class FlowTrajectory:
    """Recorded flow (fixed capacity, ``count`` valid rows; s unwrapped)."""

    s: Any
    t: Any
    length: Any
    energy: Any
    count: Any


@dataclasses.dataclass
class FlowResult:
    """Final state of a gradient flow (t: flow time, length: arclength)."""

    s: Any
    energy: Any
    t: Any
    length: Any
    dt: Any
    n_steps: Any
    n_evals: Any
    status: Any
    trajectory: Optional[FlowTrajectory]


def _validate(s0: Any, basis: np.ndarray, settings: FlowSettings) -> None:
    """Raise on bad inputs before any device work (``flow.py:_validate``)."""
    require_float64(s0, "s0")
    if s0.ndim not in (2, 3) or basis.shape != (s0.shape[-1], s0.shape[-1]):
        raise ValueError(f"s0 must be (n, d) or (b, n, d) with a (d, d) basis, got {s0.shape}")
    positive = (settings.atol, settings.rtol, settings.dt_init, settings.max_steps)
    if not all(x > 0 for x in positive):
        raise ValueError("atol, rtol, dt_init and max_steps must be positive")
    if settings.parametrization not in ("time", "arclength"):
        raise ValueError(f"unknown parametrization {settings.parametrization!r}")
    if settings.method not in ("dopri5", "rosenbrock"):
        raise ValueError(f"unknown method {settings.method!r}")
    if settings.method == "rosenbrock" and settings.parametrization != "time":
        raise ValueError("method='rosenbrock' integrates the time parametrization")
    if settings.parametrization == "arclength" and math.isfinite(settings.t_max):
        raise ValueError("t_max is supported only with parametrization='time'")
    if settings.record_every < 0 or settings.max_records < 0:
        raise ValueError("record_every and max_records must be >= 0")
    if (settings.record_every > 0) != (settings.max_records > 1):
        raise ValueError("recording needs record_every > 0 and max_records >= 2")


def gradient_flow(energy: Any, s0: Any, basis: Any, settings: FlowSettings,
                  dt0: Any = None) -> FlowResult:  # fmt: skip
    """Integrate dr/dt = -grad_r Phi from ``s0`` (fractional) until a stop.

    ``s0`` is (n, d) or a (b, n, d) batch; results have the matching leading
    axis (scalars are 0-d for an (n, d) input). Positions are not wrapped.
    ``dt0`` overrides ``settings.dt_init`` (scalar or one per lane) to resume
    a flow from ``FlowResult.dt``. NumPy in, NumPy out; CUDA tensors stay on
    the device (dopri5).
    """
    import torch

    from xla_cco.energy import StealthyEnergy

    basis = np.asarray(basis.cpu() if isinstance(basis, torch.Tensor) else basis, dtype=np.float64)
    _validate(s0, basis, settings)
    if not isinstance(energy, StealthyEnergy):
        raise TypeError("the B200 flow evaluates a StealthyEnergy on the device")
    _native.require_gpu()
    if settings.method == "rosenbrock":
        return _rosenbrock(energy, s0, basis, settings, dt0)
    single = s0.ndim == 2
    host = not (isinstance(s0, torch.Tensor) and s0.is_cuda)
    if isinstance(s0, torch.Tensor):
        s_dev = s0.detach().to("cuda", torch.float64).contiguous()
    else:
        s_dev = torch.from_numpy(np.ascontiguousarray(np.asarray(s0))).cuda()
    if single:
        s_dev = s_dev[None]
    b, n, d = s_dev.shape
    dev = s_dev.device
    index = dev.index if dev.index is not None else torch.cuda.current_device()
    h = energy.problem_handle(index, n)
    handles = (_native.ctypes.c_void_p * b)(*([h] * b))
    bases = np.ascontiguousarray(np.broadcast_to(basis, (b, d, d)))
    dt0_arr = None
    if dt0 is not None:
        dt0_arr = np.ascontiguousarray(np.broadcast_to(np.asarray(
            dt0.cpu() if isinstance(dt0, torch.Tensor) else dt0, dtype=np.float64), (b,)))
    f64, i64 = torch.float64, torch.int64
    out = {k: torch.empty(b, dtype=f64, device=dev) for k in ("energy", "t", "length", "dt")}
    out.update({k: torch.empty(b, dtype=i64, device=dev) for k in ("n_steps", "n_evals", "status")})
    out["s"] = torch.empty_like(s_dev)
    rec = settings.record_every > 0
    cap = int(settings.max_records)
    if rec:
        out["traj_s"] = torch.zeros((b, cap, n, d), dtype=f64, device=dev)
        for k in ("traj_t", "traj_length", "traj_energy"):
            out[k] = torch.zeros((b, cap), dtype=f64, device=dev)
        out["traj_count"] = torch.zeros(b, dtype=i64, device=dev)
    co = _native.FlowOutC()
    for k, t in out.items():
        setattr(co, k, t.data_ptr())
    cs = _native.FlowSettingsC(
        float(settings.rtol), float(settings.atol), float(settings.dt_init), float(settings.dt_min),
        float(settings.dt_max), float(settings.t_max), int(settings.max_steps),
        float(settings.energy_tol), float(settings.grad_tol),
        1 if settings.parametrization == "arclength" else 0, 0, int(settings.record_every),
        int(settings.max_records),
    )  # fmt: skip
    lib = _native.load()
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        code = lib.cco_gradient_flow(
            handles, stream, b, s_dev.data_ptr(), bases.ctypes.data,
            dt0_arr.ctypes.data if dt0_arr is not None else None,
            _native.ctypes.byref(cs), _native.ctypes.byref(co),
        )  # fmt: skip
    if code == _native.CCO_ERR_ROUNDS:
        raise RuntimeError("gradient flow did not finish within the round bound")
    _native.check(code, "cco_gradient_flow")
    conv = (lambda t: t.cpu().numpy()) if host else (lambda t: t)
    pick = (lambda x: x[0]) if single else (lambda x: x)
    traj = None
    if rec:
        traj = FlowTrajectory(
            s=pick(conv(out["traj_s"])), t=pick(conv(out["traj_t"])),
            length=pick(conv(out["traj_length"])), energy=pick(conv(out["traj_energy"])),
            count=pick(conv(out["traj_count"])),
        )  # fmt: skip
    return FlowResult(
        s=pick(conv(out["s"])), energy=pick(conv(out["energy"])), t=pick(conv(out["t"])),
        length=pick(conv(out["length"])), dt=pick(conv(out["dt"])),
        n_steps=pick(conv(out["n_steps"])), n_evals=pick(conv(out["n_evals"])),
        status=pick(conv(out["status"])), trajectory=traj,
    )  # fmt: skip


# ------------------------------------------------------------------ ROS2
def _rosenbrock(energy: Any, s0: Any, basis: np.ndarray, settings: FlowSettings,
                dt0: Any) -> FlowResult:  # fmt: skip
    """ROS2 (Verwer et al. 1999) with the exact Hessian, one lane at a time.

    (I - g h J) k1 = v(y), (I - g h J) k2 = v(y + h k1) - 2 k1,
    y+ = y + 3/2 h k1 + 1/2 h k2 with g = 1 + 1/sqrt(2); the error estimate
    h (k1 + k2) / 2 is filtered by (I - g h J)^-1 (Shampine), order 2 in the
    controller. The Hessian is the closed form on the GPU (DGEMM), the solves
    use an LU factorisation on the GPU.
    """
    import torch

    x = np.asarray(s0.cpu() if isinstance(s0, torch.Tensor) else s0, dtype=np.float64)
    if x.ndim == 3:
        lanes = [_rosenbrock(energy, x[i], basis, settings,
                             None if dt0 is None else np.broadcast_to(np.asarray(dt0), (x.shape[0],))[i])
                 for i in range(x.shape[0])]  # fmt: skip
        stack = lambda f: np.stack([getattr(r, f) for r in lanes])  # noqa: E731
        traj = None
        if settings.record_every > 0:
            traj = FlowTrajectory(*(np.stack([getattr(r.trajectory, f) for r in lanes])
                                    for f in ("s", "t", "length", "energy", "count")))  # fmt: skip
        return FlowResult(*(stack(f) for f in ("s", "energy", "t", "length", "dt", "n_steps",
                                                 "n_evals", "status")), trajectory=traj)  # fmt: skip
    dev = torch.device("cuda", torch.cuda.current_device())
    n, d = x.shape
    B = torch.from_numpy(basis).to(dev)
    minv = torch.linalg.inv(B @ B.T)
    binv_t = torch.linalg.inv(B).T
    eye = torch.eye(n * d, dtype=torch.float64, device=dev)

    def velocity(s):
        phi, grad, _, _ = energy.evaluate(s[None].contiguous())
        g = grad[0]
        return float(phi[0]), g, -g @ minv, float(torch.sqrt(torch.sum((g @ binv_t) ** 2)))

    def scaled_err(err_s, step):
        move = torch.sqrt(torch.mean((step @ B) ** 2))
        return float(torch.sqrt(torch.mean((err_s @ B) ** 2)) / (settings.atol + settings.rtol * move))

    def status(f, g, gn, t, dt, steps, tries):
        code = STATUS_STEP_FLOOR if dt < settings.dt_min else STATUS_RUNNING
        if t >= settings.t_max or steps >= settings.max_steps or tries >= 4 * settings.max_steps:
            code = STATUS_BUDGET
        if bool(torch.all(g == 0.0)) or gn < settings.grad_tol:
            code = STATUS_GRAD_TOL
        return STATUS_ENERGY_TOL if f < settings.energy_tol else code

    s = torch.from_numpy(x).to(dev)
    f, g, v, gn = velocity(s)
    dt = min(settings.dt_init if dt0 is None else float(dt0), settings.dt_max)
    t = length = 0.0
    steps = tries = 0
    evals = 1
    rec = settings.record_every > 0
    rows = max(settings.max_records, 1)
    rs, rt, rl, re = [x.copy()], [0.0], [0.0], [f]
    st = status(f, g, gn, t, dt, steps, tries)
    while st == STATUS_RUNNING:
        h = min(dt, settings.t_max - t)
        hess = torch.as_tensor(energy.hessian(s), device=dev).reshape(n, d, n, d)
        jac = -torch.einsum("ibjc,ba->iajc", hess, minv).reshape(n * d, n * d)
        lu, piv = torch.linalg.lu_factor(eye - _ROS_GAMMA * h * jac)
        solve = lambda r: torch.linalg.lu_solve(lu, piv, r.reshape(-1, 1)).reshape(n, d)  # noqa: E731
        k1 = solve(v)
        _, _, v1, _ = velocity(s + h * k1)
        k2 = solve(v1 - 2.0 * k1)
        s_new = s + h * (1.5 * k1 + 0.5 * k2)
        f_new, g_new, v_new, gn_new = velocity(s_new)
        chord = float(torch.sqrt(torch.sum(((s_new - s) @ B) ** 2)))
        err = scaled_err(solve(0.5 * h * (k1 + k2)), s_new - s)
        accept = err <= 1.0
        factor = min(max(_SAFETY * err ** (-1.0 / 2.0), _SHRINK_MIN), _GROW_MAX) if err > 0 else _GROW_MAX
        if not math.isfinite(factor):
            factor = _SHRINK_MIN
        dt = min(h * factor, settings.dt_max)
        if accept:
            s, f, g, v, gn = s_new, f_new, g_new, v_new, gn_new
            t += h
            length += chord
            steps += 1
        tries += 1
        evals += 2
        st = status(f, g, gn, t, dt, steps, tries)
        if accept and rec and steps % settings.record_every == 0 and len(rs) < rows:
            rs.append(s.cpu().numpy())
            rt.append(t)
            rl.append(length)
            re.append(f)
    traj = None
    if rec:
        last_final = rl[-1] == length and rt[-1] == t
        if not last_final:
            if len(rs) < rows:
                rs.append(None), rt.append(0.0), rl.append(0.0), re.append(0.0)
        rs[-1], rt[-1], rl[-1], re[-1] = s.cpu().numpy(), t, length, f
        cnt = len(rs)
        pad = rows - cnt
        traj = FlowTrajectory(
            s=np.concatenate([np.stack(rs), np.zeros((pad, n, d))]),
            t=np.array(rt + [0.0] * pad), length=np.array(rl + [0.0] * pad),
            energy=np.array(re + [0.0] * pad), count=np.asarray(cnt),
        )  # fmt: skip
    return FlowResult(s=s.cpu().numpy(), energy=np.asarray(f), t=np.asarray(t),
                      length=np.asarray(length), dt=np.asarray(dt), n_steps=np.asarray(steps),
                      n_evals=np.asarray(evals), status=np.asarray(st),
                      trajectory=traj)  # fmt: skip
