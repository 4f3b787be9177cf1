"""MD driver: tracked waves, lane initialisation, segments, chunked simulation.

Mirrors ``src/xla_cco/dynamics/run.py:112-702`` of the reference (same
names, arguments, state fields and errors). The per-step work - the
integrator, the densities of the tracked waves, centre-of-mass correction,
winding, running sums, drift guard, snapshots and the rho trace - runs in
the MD tick on the device (``cco_md_segment``): one call advances every lane
of a chunk. The host side is bookkeeping of the batched ``MDState``.

Per step (``_step`` there): integrate; densities: the constrained waves from
the force pass, the others fresh on steps divisible by ``wind_every`` (else
they keep their last value and do not wind); exp(-i k . R_cm) unless the
scheme is "verlet"; winding_update; sums of KE, Phi, Phi^2 and
|rho|^2 / N per wave; plain Verlet stops a lane with STATUS_DRIFT when
|E - e0| > drift_tol d (N - 1) T / 2; snapshots at ``record_steps``, trace
rows every ``record_rho_every`` steps. ``begin_segment`` with
``reset_winding`` marks rho_prev pending (NaN): the next device call
recomputes it from the current positions before the first step.
"""

from __future__ import annotations

import ctypes
import dataclasses
import math
import time
from pathlib import Path
from typing import Any, Dict, Optional, Sequence

import numpy as np

from xla_cco import _native
from xla_cco._types import require_float64
from xla_cco.dynamics.checkpoint import save_state
from xla_cco.dynamics.integrators import make_force_fn
from xla_cco.dynamics.state import (
    ANDERSEN_MODES,
    SCHEMES,
    MDResult,
    MDSettings,
    MDState,
    RhoTrace,
    Snapshots,
    Waves,
)
from xla_cco.dynamics.thermal import kinetic_energy, require_key
from xla_cco.kvectors import enumerate_kvectors
from xla_cco.minimize.result import STATUS_RUNNING

__all__ = ["make_waves", "make_force_fn", "init_state", "begin_segment", "md_chunk", "simulate",
           "select_dt", "MAX_RECORD_STEPS"]  # fmt: skip

MAX_RECORD_STEPS = 256
CHECKPOINT_SOURCE = "xla_cco.dynamics.run.simulate"


# ------------------------------------------------------------------ validation
def _check_settings(s: MDSettings) -> None:
    if s.scheme not in SCHEMES or s.andersen_mode not in ANDERSEN_MODES:
        raise ValueError(f"unknown scheme {s.scheme!r} or mode {s.andersen_mode!r}")
    if not (math.isfinite(s.dt) and s.dt > 0.0):
        raise ValueError(f"dt must be finite and positive, got {s.dt}")
    if not (0.0 <= s.andersen_p <= 1.0) or not (0.0 <= s.gamma < math.inf):
        raise ValueError(f"need 0 <= andersen_p <= 1 and gamma >= 0: {s}")
    if s.chunk_steps < 1 or s.wind_every < 1:
        raise ValueError("chunk_steps and wind_every must be >= 1")
    rs = tuple(s.record_steps)
    if len(rs) > MAX_RECORD_STEPS or any(int(x) != x or x < 1 for x in rs):
        raise ValueError(f"record_steps: at most {MAX_RECORD_STEPS} integers >= 1")
    if any(b <= a for a, b in zip(rs, rs[1:])):
        raise ValueError("record_steps must be strictly increasing")
    if s.record_rho_every < 0 or s.max_rho_records < 0:
        raise ValueError("record_rho_every and max_rho_records must be >= 0")
    if s.record_rho_every > 0 and s.max_rho_records < 1:
        raise ValueError("a rho trace (record_rho_every > 0) needs max_rho_records")
    if not (s.phase_floor >= 0.0) or not (s.drift_tol > 0.0):
        raise ValueError("need phase_floor >= 0 and drift_tol > 0")


def _check_lane(state: MDState, waves: Waves, settings: MDSettings) -> None:
    """Shapes of one lane's (or a batch's trailing) buffers against waves and settings."""
    w = int(waves.kvec.shape[0])
    if state.r.shape[-1:] == () or state.rho_prev.shape[-2:] != (w, 2):
        raise ValueError(f"need ({w}, 2) rho per lane, got {state.rho_prev.shape}")
    if state.snap.step.shape[-1:] != (len(settings.record_steps),):
        raise ValueError(f"snapshot capacity {state.snap.step.shape} != "
                         f"{len(settings.record_steps)} record_steps")  # fmt: skip
    if state.trace.rho.shape[-3:-1] != (settings.max_rho_records, w):
        raise ValueError(f"trace capacity {state.trace.rho.shape} != "
                         f"({settings.max_rho_records}, {w})")  # fmt: skip


def _constrained_rows(energy: Any, waves: Waves) -> np.ndarray:
    """Problem rows of the constrained waves, which must be the energy's first
    n_constrained n_vectors (their densities come from the force pass)."""
    e, w = np.asarray(energy.n_vectors), np.asarray(waves.n_vectors)
    nc = int(waves.n_constrained)
    if not (w.ndim == 2 and 1 <= nc <= w.shape[0]):
        raise ValueError("waves must hold at least the constrained rows")
    if e.ndim != 2 or e.shape[0] < nc or e.shape[1] != w.shape[1]:
        raise ValueError(f"energy n_vectors {e.shape} cannot hold the {nc} constrained waves "
                         f"of dimension {w.shape[1]}")  # fmt: skip
    if not np.array_equal(e[:nc], w[:nc]):
        raise ValueError(f"the {nc} constrained waves differ from the energy's first {nc} "
                         "n_vectors (use one k-set)")  # fmt: skip
    rows = energy._rows
    idx = np.searchsorted(rows, np.arange(nc))
    if np.any(idx >= rows.size) or not np.array_equal(rows[np.minimum(idx, rows.size - 1)], np.arange(nc)):
        raise ValueError("a constrained wave is a zero (padding) row of the energy")
    return idx.astype(np.int32)


# ------------------------------------------------------------------ waves
def make_waves(basis: np.ndarray, k_constraint: float, k_track: float) -> Waves:
    """The constrained set (|k| < k_constraint, k-set order) then the waves
    with k_constraint < |k| < k_track by |k| (both cutoffs strict);
    kvec = n 2 pi B^-T. ``ValueError`` unless 0 < k_constraint <= k_track <
    inf or when no wave lies below k_constraint."""
    b = np.asarray(basis, dtype=np.float64)
    if not (0.0 < k_constraint <= k_track < math.inf):
        raise ValueError(f"need 0 < k_constraint <= k_track < inf, got {k_constraint}, {k_track}")
    inner = enumerate_kvectors(b, 0.0, k_constraint)
    if inner.n.shape[0] == 0:
        raise ValueError(f"no constrained wave with |k| < {k_constraint}")
    blocks = [inner.n]
    if k_track > k_constraint:
        blocks.append(enumerate_kvectors(b, k_constraint, k_track).n)
    n_vec = np.concatenate(blocks).astype(np.float64)
    m = int(inner.n.shape[0])
    return Waves(n_vectors=n_vec, kvec=n_vec @ (2.0 * math.pi * np.linalg.inv(b).T),
                 constrained=np.arange(n_vec.shape[0]) < m, n_constrained=m)  # fmt: skip


# ------------------------------------------------------------------ state
def _batch(x: Any) -> Any:
    return x[None] if hasattr(x, "shape") else np.asarray(x)[None]


def _unbatch(state: MDState) -> MDState:
    def cut(obj):
        return dataclasses.replace(obj, **{f.name: getattr(obj, f.name)[0]
                                           for f in dataclasses.fields(obj)})  # fmt: skip
    out = {f.name: getattr(state, f.name)[0] for f in dataclasses.fields(state)
           if f.name not in ("snap", "trace")}  # fmt: skip
    return MDState(**out, snap=cut(state.snap), trace=cut(state.trace))


def _as_batch(state: MDState) -> MDState:
    def add(obj):
        return dataclasses.replace(obj, **{f.name: _batch(getattr(obj, f.name))
                                           for f in dataclasses.fields(obj)})  # fmt: skip
    out = {f.name: _batch(getattr(state, f.name)) for f in dataclasses.fields(state)
           if f.name not in ("snap", "trace")}  # fmt: skip
    return MDState(**out, snap=add(state.snap), trace=add(state.trace))


def _empty_buffers(b: int, n: int, d: int, w: int, settings: MDSettings):
    R, Q = len(settings.record_steps), settings.max_rho_records
    snap = Snapshots(step=np.full((b, R), -1, np.int64), time=np.zeros((b, R)),
                     wind_abs=np.zeros((b, R, w)), wind_net=np.zeros((b, R, w)),
                     rho=np.zeros((b, R, w, 2)), r=np.zeros((b, R, n, d)), phi=np.zeros((b, R)),
                     kinetic=np.zeros((b, R)), count=np.zeros(b, np.int64))  # fmt: skip
    trace = RhoTrace(rho=np.zeros((b, Q, w, 2)), time=np.zeros((b, Q)), count=np.zeros(b, np.int64))
    return snap, trace


def init_state(energy: Any, waves: Waves, basis: Any, r0: Any, v0: Any, temperature: Any,
               key: Any, settings: MDSettings) -> MDState:  # fmt: skip
    """Lane(s) at step 0: forces, rho_prev, zero winding and sums, empty buffers,
    e0 = Phi + KE(v0) (velocities as given). ``r0`` (n, d) gives one lane;
    (b, n, d) with ``temperature`` (b,) and ``key`` (b, 2) gives a batch.
    ``ValueError`` on invalid settings or shapes or constrained waves that are
    not the energy's first n_vectors; ``TypeError`` on non-float64 arrays or a
    bad key."""
    _check_settings(settings)
    require_float64(r0, "r0")
    require_float64(v0, "v0")
    on_dev = hasattr(r0, "is_cuda") and bool(r0.is_cuda)
    host = lambda x: x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)  # noqa: E731
    r0, v0, temperature, key = host(r0), host(v0), host(temperature), host(key)
    single = r0.ndim == 2
    if single:
        require_key(np.asarray(key))
    else:
        k = np.asarray(key)
        if k.dtype != np.uint32 or k.shape != (r0.shape[0], 2):
            raise TypeError("key must be uint32 of shape (2,) per lane")
    if r0.ndim not in (2, 3) or v0.shape != r0.shape:
        raise ValueError(f"r0 and v0 must share an (n, d) shape: {r0.shape}, {v0.shape}")
    rb, vb = (r0[None], v0[None]) if single else (r0, v0)
    b, n, d = rb.shape
    w = int(waves.kvec.shape[0])
    if waves.kvec.shape != (w, d):
        raise ValueError(f"waves have dimension {waves.kvec.shape}, positions {d}")
    _constrained_rows(energy, waves)
    snap, trace = _empty_buffers(b, n, d, w, settings)
    zf = np.zeros(b)
    st = MDState(
        r=rb.astype(np.float64), v=vb.astype(np.float64), f=np.zeros_like(rb), phi=np.full(b, np.nan),
        temperature=np.broadcast_to(np.asarray(temperature, np.float64), (b,)).copy(),
        key=np.asarray(key, np.uint32).reshape(b, 2).copy(), step=np.zeros(b, np.int64),
        time=zf.copy(), reset_acc=zf.copy(), rho_prev=np.full((b, w, 2), np.nan),
        wind_abs=np.zeros((b, w)), wind_net=np.zeros((b, w)), n_valid=np.zeros((b, w), np.int64),
        e0=np.full(b, np.nan), max_drift=zf.copy(), sum_kinetic=zf.copy(), sum_phi=zf.copy(),
        sum_phi2=zf.copy(), sum_s=np.zeros((b, w)), n_sum=np.zeros(b, np.int64),
        status=np.full(b, STATUS_RUNNING, np.int64), snap=snap, trace=trace,
    )  # fmt: skip
    dev = _to_device(st)
    _run_device(energy, waves, basis, settings, dev, 0)
    out = _from_device(dev, to_host=not on_dev)
    return _unbatch(out) if single else out


def begin_segment(state: MDState, settings: MDSettings, reset_sums: bool,
                  reset_winding: bool) -> MDState:  # fmt: skip
    """Start a segment: optional COM momentum removal (``settings.remove_com``),
    e0 = Phi + KE, max_drift = 0, optional reset of the sums and of the winding
    (rho_prev then pending: recomputed before the next step). Lanes whose
    status is not STATUS_RUNNING are returned unchanged. NumPy or CUDA-tensor
    states; the result is of the same kind."""
    if _on_device(state):
        import torch as xp

        mean = lambda x: x.mean(dim=-2, keepdim=True)  # noqa: E731
        ke = lambda v: 0.5 * (v * v).sum(dim=(-2, -1))  # noqa: E731
        zeros, full = xp.zeros_like, lambda x, val: xp.full_like(x, val)  # noqa: E731
    else:
        xp = np
        mean = lambda x: np.mean(x, axis=-2, keepdims=True)  # noqa: E731
        ke = kinetic_energy
        zeros, full = np.zeros_like, lambda x, val: np.full_like(x, val)  # noqa: E731
    run = state.status == STATUS_RUNNING

    def pick(new, old):
        m = run.reshape(tuple(run.shape) + (1,) * (old.ndim - run.ndim))
        return xp.where(m, new, old)

    v = state.v - mean(state.v) if settings.remove_com else state.v
    out = dataclasses.replace(state)
    out.v = pick(v, state.v)
    out.e0 = pick(state.phi + ke(out.v), state.e0)
    out.max_drift = pick(zeros(state.max_drift), state.max_drift)
    if reset_sums:
        for name in ("sum_kinetic", "sum_phi", "sum_phi2", "sum_s", "n_sum"):
            old = getattr(state, name)
            setattr(out, name, pick(zeros(old), old))
    if reset_winding:
        for name in ("wind_abs", "wind_net", "n_valid"):
            old = getattr(state, name)
            setattr(out, name, pick(zeros(old), old))
        out.rho_prev = pick(full(state.rho_prev, float("nan")), state.rho_prev)
    return out


# ------------------------------------------------------------------ device segment
_SCHEME_C = {"verlet": (0, 0), "andersen": (0, None), "baoab": (1, 0)}


def _on_device(state: MDState) -> bool:
    r = state.r
    return hasattr(r, "is_cuda") and bool(r.is_cuda)


def _fields(state: MDState) -> Dict[str, Any]:
    out: Dict[str, Any] = {}
    for f in dataclasses.fields(state):
        v = getattr(state, f.name)
        if f.name in ("snap", "trace"):
            for g in dataclasses.fields(v):
                out[f"{f.name}_{g.name}"] = getattr(v, g.name)
        else:
            out["keys" if f.name == "key" else f.name] = v
    return out


def _to_device(state: MDState) -> Dict[str, Any]:
    """Device copies of every array (uint32 keys travel as int32 bits)."""
    import torch

    dev: Dict[str, Any] = {}
    for k, v in _fields(state).items():
        if isinstance(v, torch.Tensor):
            dev[k] = v.detach().to("cuda").contiguous().clone()
        else:
            a = np.ascontiguousarray(np.asarray(v))
            dev[k] = torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda()
    return dev


def _from_device(dev: Dict[str, Any], to_host: bool) -> MDState:
    vals = {k: (t.cpu().numpy() if to_host else t) for k, t in dev.items()}
    if to_host:
        vals["keys"] = vals["keys"].view(np.uint32)
    snap = Snapshots(**{g.name: vals[f"snap_{g.name}"] for g in dataclasses.fields(Snapshots)})
    trace = RhoTrace(**{g.name: vals[f"trace_{g.name}"] for g in dataclasses.fields(RhoTrace)})
    plain = {f.name: vals["keys" if f.name == "key" else f.name] for f in dataclasses.fields(MDState)
             if f.name not in ("snap", "trace")}  # fmt: skip
    return MDState(**plain, snap=snap, trace=trace)


def _run_device(energy: Any, waves: Waves, basis: Any, settings: MDSettings, dev: Dict[str, Any],
                n_steps: int) -> None:  # fmt: skip
    """One ``cco_md_segment`` call over the device arrays ``dev`` (updated in place)."""
    import torch

    _native.require_gpu()
    b, n, d = dev["r"].shape
    w = int(waves.kvec.shape[0])
    bm = np.ascontiguousarray(np.asarray(basis, dtype=np.float64))
    if bm.shape != (d, d):
        raise ValueError(f"basis must have shape ({d}, {d}), got {bm.shape}")
    nv = np.ascontiguousarray(np.asarray(waves.n_vectors, dtype=np.float64))
    kv = np.ascontiguousarray(np.asarray(waves.kvec, dtype=np.float64))
    if not np.array_equal(nv, np.rint(nv)):
        raise ValueError("wave n_vectors must be integer-valued")
    if not np.allclose(kv, nv @ (2.0 * math.pi * np.linalg.inv(bm).T), rtol=1e-9, atol=1e-12):
        raise ValueError("waves.kvec must equal n_vectors 2 pi B^-T for this basis")
    rows = _constrained_rows(energy, waves)
    idx = dev["r"].device.index
    h = energy.problem_handle(idx if idx is not None else torch.cuda.current_device(), n)
    scheme, mode = _SCHEME_C[settings.scheme]
    if mode is None:
        mode = 1 if settings.andersen_mode == "count" else 2
    rec = np.ascontiguousarray(np.asarray(settings.record_steps, dtype=np.int64))
    cs = _native.MdSegmentSettingsC(
        float(settings.dt), float(settings.gamma), float(settings.andersen_p),
        float(settings.drift_tol), float(settings.phase_floor), int(n_steps), scheme, mode,
        int(settings.wind_every), int(rec.size), rec.ctypes.data if rec.size else None,
        int(settings.record_rho_every), int(settings.max_rho_records),
    )  # fmt: skip
    cw = _native.MdWavesC(w, int(waves.n_constrained), nv.ctypes.data, kv.ctypes.data,
                          rows.ctypes.data)  # fmt: skip
    cst = _native.MdStateC()
    for name in _native.MD_STATE_FIELDS:
        setattr(cst, name, dev[name].data_ptr())
    ticks = ctypes.c_int64(0)
    with torch.cuda.device(dev["r"].device):
        stream = torch.cuda.current_stream().cuda_stream
        code = _native.load().cco_md_segment(h, stream, b, bm.ctypes.data, ctypes.byref(cs),
                                             ctypes.byref(cw), ctypes.byref(cst), ctypes.byref(ticks))  # fmt: skip
    _native.check(code, "cco_md_segment")


def _segment(energy: Any, waves: Waves, basis: Any, settings: MDSettings, state: MDState,
             n_steps: int) -> MDState:  # fmt: skip
    """One device call over a batched state; the result is of the state's kind."""
    dev = _to_device(state)
    _run_device(energy, waves, basis, settings, dev, n_steps)
    return _from_device(dev, to_host=not _on_device(state))


def md_chunk(energy: Any, waves: Waves, basis: Any, settings: MDSettings, state: MDState,
             n_steps: int) -> MDState:  # fmt: skip
    """Advance one lane (or a batch) by min(settings.chunk_steps, n_steps) steps.

    Lanes that are not STATUS_RUNNING (or stop on a drift) keep their state
    from then on; pending rho_prev rows are recomputed first."""
    _check_settings(settings)
    single = len(tuple(state.step.shape)) == 0
    st = _as_batch(state) if single else state
    _check_lane(st, waves, settings)
    out = _segment(energy, waves, basis, settings, st, min(int(settings.chunk_steps), int(n_steps)))
    return _unbatch(out) if single else out


def _write(path: Path, state: MDState, done: int, n_steps: int) -> None:
    save_state(Path(path), state, {"source": CHECKPOINT_SOURCE, "steps_done": done,
                                   "n_steps": n_steps})  # fmt: skip


def simulate(energy: Any, waves: Waves, basis: Any, settings: MDSettings, state: MDState,
             n_steps: int, checkpoint: Optional[Path] = None,
             checkpoint_every_s: float = 1800.0) -> MDResult:  # fmt: skip
    """Run the batched lanes for ``n_steps`` steps in device calls of
    ``settings.chunk_steps``; stops early when no lane runs. With
    ``checkpoint`` the state is written there (atomically) whenever
    ``checkpoint_every_s`` seconds have passed after a chunk, and at the end.
    ``step`` is absolute; snapshots and the trace persist across calls.
    ``ValueError`` on invalid settings, an unbatched state, buffers that do not
    match the settings, constrained waves that are not the energy's first
    n_vectors, n_steps < 0 or checkpoint_every_s <= 0."""
    _check_settings(settings)
    if len(tuple(state.step.shape)) != 1:
        raise ValueError(f"state must be batched (leading lane axis), got step shape "
                         f"{tuple(state.step.shape)}")  # fmt: skip
    if int(n_steps) != n_steps or n_steps < 0 or not checkpoint_every_s > 0.0:
        raise ValueError(f"need n_steps >= 0 and checkpoint_every_s > 0, got {n_steps}, "
                         f"{checkpoint_every_s}")  # fmt: skip
    if state.step.shape[0] < 1:
        raise ValueError("need at least one lane")
    _check_lane(state, waves, settings)
    _constrained_rows(energy, waves)
    host = not _on_device(state)
    dev = _to_device(state)
    done, last = 0, time.monotonic()
    while done < n_steps and bool((dev["status"] == STATUS_RUNNING).any()):
        n_this = min(settings.chunk_steps, int(n_steps) - done)
        _run_device(energy, waves, basis, settings, dev, n_this)
        done += n_this
        if checkpoint is not None and done < n_steps and time.monotonic() - last >= checkpoint_every_s:
            _write(checkpoint, _from_device(dev, True), done, int(n_steps))
            last = time.monotonic()
    state = _from_device(dev, to_host=host)
    if checkpoint is not None:
        _write(checkpoint, state if host else _from_device(dev, True), done, int(n_steps))
    trace = state.trace if settings.record_rho_every > 0 else None
    return MDResult(state=state, snapshots=state.snap, trace=trace)


def select_dt(energy: Any, waves: Waves, basis: Any, state: MDState, ladder: Sequence[float],
              n_steps: int, drift_rel: float) -> float:  # fmt: skip
    """Largest dt of ``ladder`` whose NVE drift |E_last - E_first| / <KE> over
    ``n_steps`` Verlet steps (lanes restarted at the state's r, v, T and key,
    no drift abort, no recording) stays below ``drift_rel`` in every lane."""
    dts = sorted({float(x) for x in ladder}, reverse=True)
    if not dts or not all(math.isfinite(x) and x > 0.0 for x in dts):
        raise ValueError(f"ladder must hold finite positive steps, got {ladder}")
    if n_steps < 1 or not drift_rel > 0.0 or len(tuple(state.step.shape)) != 1:
        raise ValueError("need n_steps >= 1, drift_rel > 0 and a batched state")
    for dt in dts:
        st = MDSettings(dt=dt, scheme="verlet", remove_com=False,
                        chunk_steps=min(int(n_steps), 10_000), drift_tol=math.inf)  # fmt: skip
        lanes = init_state(energy, waves, basis, state.r, state.v, state.temperature, state.key, st)
        out = simulate(energy, waves, basis, st, lanes, int(n_steps)).state
        h = lambda x: x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)  # noqa: E731
        e_last = h(out.phi) + kinetic_energy(h(out.v))
        ke = h(out.sum_kinetic) / np.maximum(h(out.n_sum), 1)
        with np.errstate(invalid="ignore", divide="ignore"):
            rel = np.abs(e_last - h(lanes.e0)) / ke
        if np.all(rel < drift_rel):
            return dt
    raise ValueError(f"no dt in {tuple(ladder)} keeps the drift below {drift_rel}")
