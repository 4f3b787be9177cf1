"""Batched relaxation on the device (drop-in for ``xla_cco.minimize.relax``).

``relax(energy, s0, settings, chunk_iters=2000)`` relaxes a (B, N, d) batch
and returns a ``RelaxResult`` with a leading lane axis, in input order
(``minimize/__init__.py:102-151``). Each lane is a device state machine
(``csrc/cco_opt.cu``); a finished lane is frozen bit-exactly and skipped by
every later launch, which is the reference's per-lane freeze plus host-side
compaction done on the device. ``chunk_iters`` is validated and accepted; the
result does not depend on it (the reference guarantees the same).
"""

from __future__ import annotations

from typing import Any, List, Sequence, Tuple, Union

import numpy as np

from xla_cco import _native
from xla_cco._types import require_float64
from xla_cco.minimize.descent import DescentSettings
from xla_cco.minimize.lbfgs import LBFGSSettings
from xla_cco.minimize.result import STATUS_BUDGET, STATUS_RUNNING, RelaxResult, Trajectory  # noqa: F401

__all__ = ["relax", "relax_device", "relax_external", "relax_mixed", "relax_mixed_device",
           "DescentSettings", "LBFGSSettings"]


def _descent_c(st: DescentSettings) -> _native.DescentSettingsC:
    return _native.DescentSettingsC(
        float(st.step_init), float(st.step_min), float(st.shrink), float(st.grow),
        float(st.rel_tol), int(st.max_evals), float(st.energy_tol), int(st.record_every),
        int(st.max_records),
    )  # fmt: skip


def _lbfgs_c(st: LBFGSSettings) -> _native.LBFGSSettingsC:
    if not 1 <= len(st.rescales) <= _native.MAX_RESCALES:
        raise ValueError(f"need 1..{_native.MAX_RESCALES} rescale passes")
    c = _native.LBFGSSettingsC()
    c.memory = int(st.memory)
    c.n_rescales = len(st.rescales)
    for i, r in enumerate(st.rescales):
        c.rescales[i] = float(r)
    c.max_evals_per_pass = int(st.max_evals_per_pass)
    c.energy_tol = float(st.energy_tol)
    c.grad_tol = float(st.grad_tol)
    c.stagnation_patience = int(st.stagnation_patience)
    c.max_linesearch_steps = int(st.max_linesearch_steps)
    c.record_every = int(st.record_every)
    c.max_records = int(st.max_records)
    if st.precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {st.precision!r}")
    c.precision = 1 if st.precision == "mixed" else 0
    return c


def _settings_c(settings: Any, mixed: bool = False):
    suffix = "_mixed" if mixed else ""
    if isinstance(settings, DescentSettings):
        return _descent_c(settings), "cco_relax_descent" + suffix
    if isinstance(settings, LBFGSSettings):
        return _lbfgs_c(settings), "cco_relax_lbfgs" + suffix
    raise TypeError(f"unsupported settings type {type(settings).__name__}")


def _outputs(b: int, s_shape: tuple, traj_s_shape: tuple, settings: Any, dev: Any) -> dict:
    import torch

    f64, i64 = torch.float64, torch.int64
    out = {
        "s": torch.empty(s_shape, dtype=f64, device=dev),
        "energy": torch.empty(b, dtype=f64, device=dev),
        "grad_norm": torch.empty(b, dtype=f64, device=dev),
        "n_evals": torch.empty(b, dtype=i64, device=dev),
        "n_iters": torch.empty(b, dtype=i64, device=dev),
        "status": torch.empty(b, dtype=i64, device=dev),
        "latency_ns": torch.empty(b, dtype=i64, device=dev),
        "n_evals_fp32": torch.zeros(b, dtype=i64, device=dev),
    }
    if settings.record_every > 0 and settings.max_records > 0:
        cap = int(settings.max_records)
        out["traj_s"] = torch.zeros(traj_s_shape, dtype=f64, device=dev)
        out["traj_energy"] = torch.zeros((b, cap), dtype=f64, device=dev)
        out["traj_step"] = torch.zeros((b, cap), dtype=f64, device=dev)
        out["traj_iteration"] = torch.zeros((b, cap), dtype=i64, device=dev)
        out["traj_count"] = torch.zeros(b, dtype=i64, device=dev)
    return out


def _call_relax(fn: str, first: Any, dev: Any, b: int, s0_ptr: int, cset: Any, chunk_iters: int,
                out: dict) -> None:  # fmt: skip
    import torch

    co = _native.RelaxOutC()
    for key in ("s", "energy", "grad_norm", "n_evals", "n_iters", "status", "latency_ns",
                "n_evals_fp32", "traj_s", "traj_energy", "traj_step", "traj_iteration",
                "traj_count"):  # fmt: skip
        if key in out:
            setattr(co, key, out[key].data_ptr())
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        code = getattr(_native.load(), fn)(
            first, stream, b, s0_ptr, _native.ctypes.byref(cset), int(chunk_iters),
            _native.ctypes.byref(co),
        )  # fmt: skip
    if code == _native.CCO_ERR_ROUNDS:
        raise RuntimeError("relax did not finish within the round bound")
    _native.check(code, fn)
    out["ticks"] = int(co.ticks)
    out["launches"] = int(co.launches)
    out["schedule"] = (int(co.branches), int(co.graph_ticks))
    out["overlap"] = bool(co.overlap)


def relax_device(energy: Any, s0: Any, settings: Union[DescentSettings, LBFGSSettings],
                 chunk_iters: int = 2_000) -> dict:  # fmt: skip
    """Run the device relaxation on a CUDA tensor ``s0`` (B, N, d); results stay on the device.

    Returns a dict of CUDA tensors (``s``, ``energy``, ``grad_norm``,
    ``n_evals``, ``n_iters``, ``status``, trajectory fields) plus ``ticks``.
    """
    import torch

    from xla_cco.energy import StealthyEnergy

    if not isinstance(energy, StealthyEnergy):
        raise TypeError("the B200 relax path evaluates a StealthyEnergy on the device")
    cset, fn = _settings_c(settings)
    if energy._zero_weight != 0.0:
        raise ValueError("zero k rows with nonzero weight are not supported by relax")
    b, n, d = s0.shape
    assert d == energy.dim, "dimension mismatch"
    dev = s0.device
    h = energy.problem_handle(dev.index if dev.index is not None else torch.cuda.current_device(), n)
    out = _outputs(b, tuple(s0.shape), (b, int(settings.max_records), n, d), settings, dev)
    _call_relax(fn, h, dev, b, s0.data_ptr(), cset, chunk_iters, out)
    return out


def _max_ticks(settings: Union[DescentSettings, LBFGSSettings]) -> int:
    """The tick bound of a relaxation (one evaluation per lane and tick): its
    evaluation budget plus a margin, like the fused path's round bound."""
    if isinstance(settings, DescentSettings):
        return 1 + settings.max_evals // 2 + 64
    per_pass = settings.max_evals_per_pass + settings.max_linesearch_steps + 1
    return 1 + len(settings.rescales) * per_pass + 64


def relax_external(energy: Any, s0: Any, settings: Union[DescentSettings, LBFGSSettings]) -> dict:
    """Relax a CUDA batch ``s0`` (B, N, d) under any ``AbstractEnergy``.

    The lanes are the device state machines of the fused path (the same
    records and update kernels, ``cco_stepper_*``); every tick this loop
    hands the lanes' probe positions to ``energy.value_and_grad`` - one call
    per lane, as the reference vmaps it, or one ``energy.value_and_grad_batch``
    call on the whole (B, N, d) batch when the energy defines it - and feeds
    the results back. FP64 only, no trajectory recording. Returns the dict of
    ``relax_device``.
    """
    import torch

    if isinstance(settings, LBFGSSettings) and settings.precision != "fp64":
        raise ValueError("mixed precision needs a StealthyEnergy (its FP32 kernels)")
    if settings.record_every > 0 and settings.max_records > 0:
        raise ValueError("trajectory recording needs a StealthyEnergy")
    cset, _ = _settings_c(settings)
    method = 0 if isinstance(settings, DescentSettings) else 1
    b, n, d = (int(x) for x in s0.shape)
    dev = s0.device
    index = dev.index if dev.index is not None else torch.cuda.current_device()
    lib = _native.load()
    batched = getattr(energy, "value_and_grad_batch", None)
    out = _outputs(b, (b, n, d), (b, 0, n, d), settings, dev)
    with torch.cuda.device(index):
        stream = torch.cuda.current_stream(index).cuda_stream
        h = _native._vp()
        _native.check(lib.cco_stepper_create(index, stream, method, _native.ctypes.byref(cset), b, n,
                                             d, s0.contiguous().data_ptr(),
                                             _native.ctypes.byref(h)), "cco_stepper_create")  # fmt: skip
        try:
            ps = torch.empty((b, n, d), dtype=torch.float64, device=dev)
            f = torch.empty(b, dtype=torch.float64, device=dev)
            g = torch.empty((b, n, d), dtype=torch.float64, device=dev)
            running = _native.ctypes.c_int64(b)
            bound, ticks = _max_ticks(settings), 0
            while running.value > 0:
                if ticks >= bound:
                    raise RuntimeError("relax did not finish within the round bound")
                _native.check(lib.cco_stepper_probes(h, stream, ps.data_ptr()), "cco_stepper_probes")
                if batched is not None:
                    fv, gv = batched(ps)
                    f.copy_(torch.as_tensor(fv, dtype=torch.float64, device=dev).reshape(b))
                    g.copy_(torch.as_tensor(gv, dtype=torch.float64, device=dev).reshape(b, n, d))
                else:
                    for i in range(b):
                        fv, gv = energy.value_and_grad(ps[i])
                        f[i] = torch.as_tensor(fv, dtype=torch.float64, device=dev)
                        g[i] = torch.as_tensor(gv, dtype=torch.float64, device=dev).reshape(n, d)
                _native.check(lib.cco_stepper_advance(h, stream, f.data_ptr(), g.data_ptr(),
                                                      _native.ctypes.byref(running)),
                              "cco_stepper_advance")  # fmt: skip
                ticks += 1
            co = _native.RelaxOutC()
            for key in ("s", "energy", "grad_norm", "n_evals", "n_iters", "status", "latency_ns",
                        "n_evals_fp32"):  # fmt: skip
                setattr(co, key, out[key].data_ptr())
            _native.check(lib.cco_stepper_finish(h, stream, _native.ctypes.byref(co)),
                          "cco_stepper_finish")  # fmt: skip
        finally:
            lib.cco_stepper_destroy(h)
    out["ticks"] = ticks
    out["launches"] = 0
    out["schedule"] = (0, 0)
    out["overlap"] = False
    return out


def relax(energy: Any, s0: Any, settings: Union[DescentSettings, LBFGSSettings],
          chunk_iters: int = 2_000) -> RelaxResult:  # fmt: skip
    """Relax a batch of configurations; result leaves carry a leading batch axis.

    ``TypeError`` if ``s0`` is not float64 or ``settings`` is of another type;
    ``RuntimeError`` if the round bound is exceeded or no GPU is visible.
    """
    import torch

    require_float64(s0, "s0")
    assert s0.ndim == 3, "s0 must have shape (b, n, d)"
    assert chunk_iters >= 1, "chunk_iters must be positive"
    assert s0.shape[0] >= 1, "need at least one configuration"
    if not isinstance(settings, (DescentSettings, LBFGSSettings)):
        raise TypeError(f"unsupported settings type {type(settings).__name__}")
    _native.require_gpu()
    if isinstance(s0, torch.Tensor):
        host = not s0.is_cuda
        # a pinned host tensor is copied asynchronously on the current stream
        s_dev = s0.cuda(non_blocking=True) if host else s0.contiguous()
    else:
        host = True
        s_dev = torch.from_numpy(np.ascontiguousarray(np.asarray(s0))).cuda()
    from xla_cco.energy import AbstractEnergy, StealthyEnergy

    if isinstance(energy, StealthyEnergy):
        out = relax_device(energy, s_dev, settings, chunk_iters)
    elif isinstance(energy, AbstractEnergy):
        out = relax_external(energy, s_dev, settings)
    else:
        raise TypeError(f"energy must be an AbstractEnergy, got {type(energy).__name__}")
    conv = (lambda t: t.cpu().numpy()) if host else (lambda t: t)
    traj = None
    if "traj_s" in out:
        traj = Trajectory(
            s=conv(out["traj_s"]), energy=conv(out["traj_energy"]), step=conv(out["traj_step"]),
            iteration=conv(out["traj_iteration"]), count=conv(out["traj_count"]),
        )  # fmt: skip
    return RelaxResult(
        s=conv(out["s"]), energy=conv(out["energy"]), grad_norm=conv(out["grad_norm"]),
        n_evals=conv(out["n_evals"]), n_iters=conv(out["n_iters"]), status=conv(out["status"]),
        trajectory=traj,
    )  # fmt: skip


def relax_mixed_device(energies: Sequence[Any], s0: Any, shapes: Sequence[Tuple[int, int]],
                       settings: Union[DescentSettings, LBFGSSettings],
                       chunk_iters: int = 2_000) -> dict:  # fmt: skip
    """One device relaxation over lanes of different problems (N, d and k-set).

    ``energies[i]`` is lane i's ``StealthyEnergy`` and ``shapes[i]`` its
    (N_i, d_i); ``s0`` is a flat CUDA float64 tensor with every lane's
    positions packed one after the other. Returns a dict of CUDA tensors:
    ``s`` packed the same way, per-lane scalars of shape (B,), ``traj_s``
    packed with ``max_records`` rows per lane, plus ``offsets`` (B + 1 element
    offsets into ``s``), ``ticks`` and ``launches``.
    """
    import torch

    from xla_cco.energy import StealthyEnergy

    cset, fn = _settings_c(settings, mixed=True)
    b = len(energies)
    if b < 1 or len(shapes) != b:
        raise ValueError("need one (N, d) shape per energy and at least one configuration")
    dev = s0.device
    index = dev.index if dev.index is not None else torch.cuda.current_device()
    handles = (_native.ctypes.c_void_p * b)()
    offsets = [0]
    for i, (en, (n, d)) in enumerate(zip(energies, shapes)):
        if not isinstance(en, StealthyEnergy):
            raise TypeError("the B200 relax path evaluates a StealthyEnergy on the device")
        if en._zero_weight != 0.0:
            raise ValueError("zero k rows with nonzero weight are not supported by relax")
        assert d == en.dim, f"lane {i}: dimension mismatch"
        handles[i] = en.problem_handle(index, int(n))
        offsets.append(offsets[-1] + int(n) * int(d))
    assert s0.numel() == offsets[-1], "s0 does not hold the packed positions of every lane"
    cap = int(settings.max_records)
    out = _outputs(b, (offsets[-1],), (cap * offsets[-1],), settings, dev)
    _call_relax(fn, handles, dev, b, s0.data_ptr(), cset, chunk_iters, out)
    out["offsets"] = offsets
    return out


def relax_mixed(energies: Sequence[Any], s0: Sequence[Any],
                settings: Union[DescentSettings, LBFGSSettings],
                chunk_iters: int = 2_000) -> List[RelaxResult]:  # fmt: skip
    """Relax instances of different N, d and k-set together in one device run.

    ``energies[i]`` and ``s0[i]`` (an (N_i, d_i) float64 array, NumPy or
    torch) form lane i. Returns one ``RelaxResult`` per lane with a batch axis
    of 1, bit-identical to ``relax(energies[i], s0[i][None], settings)``.
    """
    import torch

    assert chunk_iters >= 1, "chunk_iters must be positive"
    if len(energies) != len(s0) or not energies:
        raise ValueError("need one initial configuration per energy and at least one")
    if not isinstance(settings, (DescentSettings, LBFGSSettings)):
        raise TypeError(f"unsupported settings type {type(settings).__name__}")
    _native.require_gpu()
    host = not (isinstance(s0[0], torch.Tensor) and s0[0].is_cuda)
    shapes = []
    for x in s0:
        require_float64(x, "s0")
        assert x.ndim == 2, "each configuration must have shape (n, d)"
        shapes.append((int(x.shape[0]), int(x.shape[1])))
    if host:
        flat = np.concatenate([np.asarray(x.cpu() if isinstance(x, torch.Tensor) else x).ravel()
                               for x in s0])  # fmt: skip
        s_dev = torch.from_numpy(flat).pin_memory().cuda(non_blocking=True)
    else:
        s_dev = torch.cat([x.reshape(-1) for x in s0])
    out = relax_mixed_device(energies, s_dev, shapes, settings, chunk_iters)
    conv = (lambda t: t.cpu().numpy()) if host else (lambda t: t)
    keys = ("s", "energy", "grad_norm", "n_evals", "n_iters", "status")
    tkeys = ("traj_s", "traj_energy", "traj_step", "traj_iteration", "traj_count")
    res = {k: conv(out[k]) for k in keys + tkeys if k in out}
    off, cap = out["offsets"], int(settings.max_records)
    results = []
    for i, (n, d) in enumerate(shapes):
        traj = None
        if "traj_s" in res:
            traj = Trajectory(
                s=res["traj_s"][cap * off[i]:cap * off[i + 1]].reshape(1, cap, n, d),
                energy=res["traj_energy"][i:i + 1], step=res["traj_step"][i:i + 1],
                iteration=res["traj_iteration"][i:i + 1], count=res["traj_count"][i:i + 1],
            )  # fmt: skip
        results.append(RelaxResult(
            s=res["s"][off[i]:off[i + 1]].reshape(1, n, d), energy=res["energy"][i:i + 1],
            grad_norm=res["grad_norm"][i:i + 1], n_evals=res["n_evals"][i:i + 1],
            n_iters=res["n_iters"][i:i + 1], status=res["status"][i:i + 1], trajectory=traj,
        ))  # fmt: skip
    return results
