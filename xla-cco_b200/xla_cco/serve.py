"""Serving pool: relaxation requests of any N, d and k-set, continuously batched.

The reference has no serving loop; it relaxes one ``(energy, batch)`` pair per
``relax`` call (``minimize/__init__.py:102-151``). ``RelaxServer`` wraps the
C serving pool (``cco_server_*`` in ``include/cco.h``): requests are queued
in arrival order and admitted onto the device while their lane records fit
the lane and HBM budgets; requests that arrive while others run join the
running set at the next graph boundary, and finished lanes leave it. Each
result is bit-identical to ``relax(energy, s0[None], settings)`` for the
same configuration alone.

    with RelaxServer(LBFGSSettings(energy_tol=1e-20)) as srv:
        t = srv.submit(energy, s0)          # s0: (N, d) float64, host
        res = srv.result(t)                 # ServedResult
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any, Optional

import numpy as np

from xla_cco import _native
from xla_cco._types import require_float64
from xla_cco.minimize import _lbfgs_c
from xla_cco.minimize.lbfgs import LBFGSSettings

__all__ = ["RelaxServer", "ServedResult", "ServerStats"]


@dataclass(frozen=True)
class ServedResult:
    """One finished request. Times are host steady-clock nanoseconds."""

    s: np.ndarray           # (N, d) final positions wrapped into [0, 1)
    energy: float
    grad_norm: float
    n_evals: int
    n_iters: int
    status: int             # STATUS_* of minimize.result, STATUS_CANCELLED included
    submit_ns: int
    admit_ns: int
    done_ns: int
    device_ns: int          # device time from the lane's first tick to its completion
    error: int              # CCO_OK, or the code of a device failure that ended it
    n_evals_fp32: int = 0   # evaluations done in FP32 (settings.precision == "mixed")

    @property
    def latency_s(self) -> float:
        """Submission to completion, seconds (queueing included)."""
        return (self.done_ns - self.submit_ns) * 1e-9


@dataclass(frozen=True)
class ServerStats:
    submitted: int
    admitted: int
    completed: int
    cancelled: int
    pending: int
    running: int
    bytes_in_use: int
    peak_bytes: int
    peak_lanes: int
    budget_bytes: int
    graphs: int
    ticks: int
    rebuilds: int


class RelaxServer:
    """A serving pool on one CUDA device with one L-BFGS setting.

    ``max_lanes`` bounds the lanes on the device at once, ``hbm_budget_bytes``
    the memory of their records (default 150 GB, clamped to 90% of the free
    device memory), ``graph_ticks`` the ticks per launched graph.
    """

    def __init__(self, settings: LBFGSSettings = LBFGSSettings(), device: int = 0,
                 max_lanes: int = 0, hbm_budget_bytes: int = 0, graph_ticks: int = 0,
                 branches: int = 0) -> None:  # fmt: skip
        self._h = ctypes.c_void_p()
        if not isinstance(settings, LBFGSSettings):
            raise TypeError("the serving pool runs L-BFGS relaxations")
        _native.require_gpu()
        self._lib = _native.load()
        self._settings = settings
        self._device = int(device)
        self._shapes: dict = {}
        cfg = _native.ServerConfigC(int(max_lanes), int(hbm_budget_bytes), int(graph_ticks),
                                    int(branches))  # fmt: skip
        cset = _lbfgs_c(settings)
        h = ctypes.c_void_p()
        _native.check(self._lib.cco_server_create(self._device, ctypes.byref(cset), ctypes.byref(cfg),
                                                  ctypes.byref(h)), "cco_server_create")  # fmt: skip
        self._h = h

    # ------------------------------------------------------------ requests
    def submit(self, energy: Any, s0: Any) -> int:
        """Queue one (N, d) float64 configuration of ``energy``; returns a ticket."""
        from xla_cco.energy import StealthyEnergy

        if not isinstance(energy, StealthyEnergy):
            raise TypeError("the serving pool evaluates a StealthyEnergy on the device")
        if energy._zero_weight != 0.0:
            raise ValueError("zero k rows with nonzero weight are not supported by relax")
        require_float64(s0, "s0")
        x = np.ascontiguousarray(np.asarray(s0.cpu() if hasattr(s0, "cpu") else s0))
        assert x.ndim == 2 and x.shape[1] == energy.dim, "s0 must have shape (n, d)"
        handle = energy.problem_handle(self._device, int(x.shape[0]))
        t = ctypes.c_int64()
        code = self._lib.cco_server_submit(self._handle(), handle, x.ctypes.data, ctypes.byref(t))
        _native.check(code, "cco_server_submit")
        self._shapes[int(t.value)] = x.shape
        return int(t.value)

    def poll(self, ticket: int, timeout_s: Optional[float] = 0.0) -> Optional[ServedResult]:
        """The result if the request is done within ``timeout_s`` (None: wait until done).

        A returned result releases the ticket.
        """
        shape = self._shapes.get(int(ticket))
        if shape is None:
            raise ValueError(f"unknown ticket {ticket}")
        s = np.empty(shape, dtype=np.float64)
        out = _native.RequestResultC()
        out.s = s.ctypes.data
        ms = -1 if timeout_s is None else int(max(timeout_s, 0.0) * 1000)
        code = self._lib.cco_server_poll(self._handle(), int(ticket), ms, ctypes.byref(out))
        if code == _native.CCO_ERR_TIMEOUT:
            return None
        _native.check(code, "cco_server_poll")
        del self._shapes[int(ticket)]
        return ServedResult(
            s=s, energy=float(out.energy), grad_norm=float(out.grad_norm), n_evals=int(out.n_evals),
            n_iters=int(out.n_iters), status=int(out.status), submit_ns=int(out.submit_ns),
            admit_ns=int(out.admit_ns), done_ns=int(out.done_ns), device_ns=int(out.device_ns),
            error=int(out.error), n_evals_fp32=int(out.n_evals_fp32),
        )  # fmt: skip

    def result(self, ticket: int) -> ServedResult:
        """Block until the request is done."""
        res = self.poll(ticket, None)
        assert res is not None
        return res

    def cancel(self, ticket: int) -> None:
        """End a queued or running request with STATUS_CANCELLED (no effect once done)."""
        _native.check(self._lib.cco_server_cancel(self._handle(), int(ticket)), "cco_server_cancel")

    def stats(self) -> ServerStats:
        st = _native.ServerStatsC()
        _native.check(self._lib.cco_server_get_stats(self._handle(), ctypes.byref(st)),
                      "cco_server_get_stats")  # fmt: skip
        return ServerStats(**{name: int(getattr(st, name)) for name, _ in st._fields_})

    # ------------------------------------------------------------ lifetime
    def close(self) -> None:
        """Cancel what is queued or running and stop the driver."""
        if self._h.value:
            self._lib.cco_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def _handle(self) -> ctypes.c_void_p:
        if not self._h.value:
            raise RuntimeError("server is closed")
        return self._h

    def __enter__(self) -> "RelaxServer":
        return self

    def __exit__(self, *exc: Any) -> None:
        self.close()

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass
