"""ctypes binding of libcco.so (the C ABI declared in include/cco.h).

The library is the only compute path: there is no CPU fallback. Loading
fails loudly if the shared object is missing, and every compute entry point
raises ``RuntimeError`` when no CUDA device is visible (the reference's
fail-fast GPU guard, ``xla_cco/_device.py:137-142``).
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libcco.so"

CCO_OK = 0
CCO_ERR_ARG = 1
CCO_ERR_OOM = 2
CCO_ERR_ADMISSION = 3
CCO_ERR_DEVICE = 4
CCO_ERR_TIMEOUT = 5
CCO_ERR_ROUNDS = 6
CCO_ERR_NODEVICE = 7
MAX_RESCALES = 8

_c_int_p = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class DescentSettingsC(ctypes.Structure):
    _fields_ = [
        ("step_init", ctypes.c_double),
        ("step_min", ctypes.c_double),
        ("shrink", ctypes.c_double),
        ("grow", ctypes.c_double),
        ("rel_tol", ctypes.c_double),
        ("max_evals", ctypes.c_int64),
        ("energy_tol", ctypes.c_double),
        ("record_every", ctypes.c_int64),
        ("max_records", ctypes.c_int64),
    ]


class LBFGSSettingsC(ctypes.Structure):
    _fields_ = [
        ("memory", ctypes.c_int64),
        ("n_rescales", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("rescales", ctypes.c_double * MAX_RESCALES),
        ("max_evals_per_pass", ctypes.c_int64),
        ("energy_tol", ctypes.c_double),
        ("grad_tol", ctypes.c_double),
        ("stagnation_patience", ctypes.c_int64),
        ("max_linesearch_steps", ctypes.c_int64),
        ("record_every", ctypes.c_int64),
        ("max_records", ctypes.c_int64),
    ]


class RelaxOutC(ctypes.Structure):
    _fields_ = [
        ("s", _vp),
        ("energy", _vp),
        ("grad_norm", _vp),
        ("n_evals", _vp),
        ("n_iters", _vp),
        ("status", _vp),
        ("traj_s", _vp),
        ("traj_energy", _vp),
        ("traj_step", _vp),
        ("traj_iteration", _vp),
        ("traj_count", _vp),
        ("latency_ns", _vp),
        ("n_evals_fp32", _vp),
        ("ticks", ctypes.c_int64),
        ("launches", ctypes.c_int64),
        ("branches", ctypes.c_int32),
        ("graph_ticks", ctypes.c_int32),
        ("overlap", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class ServerConfigC(ctypes.Structure):
    _fields_ = [
        ("max_lanes", ctypes.c_int64),
        ("hbm_budget_bytes", ctypes.c_int64),
        ("graph_ticks", ctypes.c_int32),
        ("branches", ctypes.c_int32),
    ]


class RequestResultC(ctypes.Structure):
    _fields_ = [
        ("s", _vp),
        ("energy", ctypes.c_double),
        ("grad_norm", ctypes.c_double),
        ("n_evals", ctypes.c_int64),
        ("n_iters", ctypes.c_int64),
        ("status", ctypes.c_int64),
        ("submit_ns", ctypes.c_int64),
        ("admit_ns", ctypes.c_int64),
        ("done_ns", ctypes.c_int64),
        ("device_ns", ctypes.c_int64),
        ("error", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("n_evals_fp32", ctypes.c_int64),
    ]


class ServerStatsC(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64) for name in (
        "submitted", "admitted", "completed", "cancelled", "pending", "running",
        "bytes_in_use", "peak_bytes", "peak_lanes", "budget_bytes", "graphs", "ticks", "rebuilds",
    )]  # fmt: skip


class FlowSettingsC(ctypes.Structure):
    _fields_ = [
        ("rtol", ctypes.c_double), ("atol", ctypes.c_double),
        ("dt_init", ctypes.c_double), ("dt_min", ctypes.c_double),
        ("dt_max", ctypes.c_double), ("t_max", ctypes.c_double),
        ("max_steps", ctypes.c_int64), ("energy_tol", ctypes.c_double),
        ("grad_tol", ctypes.c_double), ("arclength", ctypes.c_int32),
        ("pad_", ctypes.c_int32), ("record_every", ctypes.c_int64),
        ("max_records", ctypes.c_int64),
    ]  # fmt: skip


class FlowOutC(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "s", "energy", "t", "length", "dt", "n_steps", "n_evals", "status", "traj_s", "traj_t",
        "traj_length", "traj_energy", "traj_count",
    )] + [("ticks", ctypes.c_int64), ("launches", ctypes.c_int64)]  # fmt: skip


class MdSettingsC(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double), ("n_steps", ctypes.c_int64), ("scheme", ctypes.c_int32),
        ("andersen", ctypes.c_int32), ("andersen_p", ctypes.c_double), ("gamma", ctypes.c_double),
        ("temperature", ctypes.c_double), ("drift_tol", ctypes.c_double),
    ]  # fmt: skip


class MdOutC(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "r", "v", "f", "energy", "kinetic", "max_drift", "n_resets", "reset_acc", "keys", "status",
    )] + [("ticks", ctypes.c_int64), ("launches", ctypes.c_int64)]  # fmt: skip


# (name, restype, argtypes) for every symbol include/cco.h declares
class MdSegmentSettingsC(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double), ("gamma", ctypes.c_double), ("andersen_p", ctypes.c_double),
        ("drift_tol", ctypes.c_double), ("phase_floor", ctypes.c_double),
        ("n_steps", ctypes.c_int64), ("scheme", ctypes.c_int32), ("andersen", ctypes.c_int32),
        ("wind_every", ctypes.c_int32), ("n_record_steps", ctypes.c_int32),
        ("record_steps", ctypes.c_void_p), ("record_rho_every", ctypes.c_int32),
        ("max_rho_records", ctypes.c_int32),
    ]  # fmt: skip


class MdWavesC(ctypes.Structure):
    _fields_ = [("n_waves", ctypes.c_int32), ("n_constrained", ctypes.c_int32),
                ("n_vectors", ctypes.c_void_p), ("kvec", ctypes.c_void_p),
                ("constrained_rows", ctypes.c_void_p)]  # fmt: skip


MD_STATE_FIELDS = (
    "r", "v", "f", "phi", "temperature", "time", "reset_acc", "e0", "max_drift", "sum_kinetic",
    "sum_phi", "sum_phi2", "keys", "step", "status", "n_sum", "rho_prev", "wind_abs", "wind_net",
    "sum_s", "n_valid", "snap_step", "snap_count", "snap_time", "snap_phi", "snap_kinetic",
    "snap_wind_abs", "snap_wind_net", "snap_rho", "snap_r", "trace_rho", "trace_time",
    "trace_count",
)


class MdStateC(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in MD_STATE_FIELDS]


SIGNATURES = {
    "cco_abi_version": (ctypes.c_int, []),
    "cco_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "cco_last_error": (ctypes.c_char_p, []),
    "cco_device_count": (ctypes.c_int, [_c_int_p]),
    "cco_problem_create": (
        ctypes.c_int,
        [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_double,
         ctypes.POINTER(_vp)],
    ),  # fmt: skip
    "cco_problem_destroy": (ctypes.c_int, [_vp]),
    "cco_problem_info": (ctypes.c_int, [_vp, _c_int_p, _c_int_p, _c_int_p, _c_int_p, _c_int_p, _c_int_p]),
    "cco_energy_grad": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
    "cco_energy_grad_noalloc": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp, _vp]),
    "cco_energy_grad_fp32": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp, _vp]),
    "cco_hessian": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp]),
    "cco_stepper_create": (
        ctypes.c_int,
        [ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
         ctypes.POINTER(_vp)],
    ),  # fmt: skip
    "cco_stepper_probes": (ctypes.c_int, [_vp, _vp, _vp]),
    "cco_stepper_advance": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_int64)]),
    "cco_stepper_finish": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(RelaxOutC)]),
    "cco_stepper_destroy": (ctypes.c_int, [_vp]),
    "cco_relax_descent": (
        ctypes.c_int,
        [_vp, _vp, ctypes.c_int, _vp, ctypes.POINTER(DescentSettingsC), ctypes.c_int,
         ctypes.POINTER(RelaxOutC)],
    ),  # fmt: skip
    "cco_relax_lbfgs": (
        ctypes.c_int,
        [_vp, _vp, ctypes.c_int, _vp, ctypes.POINTER(LBFGSSettingsC), ctypes.c_int,
         ctypes.POINTER(RelaxOutC)],
    ),  # fmt: skip
    "cco_schedule_reset": (ctypes.c_int, []),
    "cco_md_run": (
        ctypes.c_int,
        [_vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(MdSettingsC),
         ctypes.POINTER(MdOutC)],
    ),  # fmt: skip
    "cco_gradient_flow": (
        ctypes.c_int,
        [_vp, _vp, ctypes.c_int, _vp, _vp, _vp, ctypes.POINTER(FlowSettingsC),
         ctypes.POINTER(FlowOutC)],
    ),  # fmt: skip
    "cco_server_create": (
        ctypes.c_int,
        [ctypes.c_int, ctypes.POINTER(LBFGSSettingsC), ctypes.POINTER(ServerConfigC),
         ctypes.POINTER(_vp)],
    ),  # fmt: skip
    "cco_pair_histogram": (
        ctypes.c_int,
        [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp,
         _vp],
    ),  # fmt: skip
    "cco_nearest_neighbor": (
        ctypes.c_int,
        [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp],
    ),  # fmt: skip
    "cco_problem_pass1_form": (ctypes.c_int, [_vp, _c_int_p]),
    "cco_md_segment": (
        ctypes.c_int,
        [_vp, _vp, ctypes.c_int, _vp, ctypes.POINTER(MdSegmentSettingsC), ctypes.POINTER(MdWavesC),
         ctypes.POINTER(MdStateC), ctypes.POINTER(ctypes.c_int64)],
    ),  # fmt: skip
    "cco_server_destroy": (ctypes.c_int, [_vp]),
    "cco_server_submit": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(ctypes.c_int64)]),
    "cco_server_poll": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(RequestResultC)]),
    "cco_server_cancel": (ctypes.c_int, [_vp, ctypes.c_int64]),
    "cco_server_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ServerStatsC)]),
    "cco_relax_descent_mixed": (
        ctypes.c_int,
        [_vp, _vp, ctypes.c_int, _vp, ctypes.POINTER(DescentSettingsC), ctypes.c_int,
         ctypes.POINTER(RelaxOutC)],
    ),  # fmt: skip
    "cco_relax_lbfgs_mixed": (
        ctypes.c_int,
        [_vp, _vp, ctypes.c_int, _vp, ctypes.POINTER(LBFGSSettingsC), ctypes.c_int,
         ctypes.POINTER(RelaxOutC)],
    ),  # fmt: skip
}

_lock = threading.Lock()
_lib = None


def load() -> ctypes.CDLL:
    """Load libcco.so once (``RuntimeError`` if it was never built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = Path(os.environ.get("CCO_LIB", LIB_PATH))
        if not path.exists():
            raise RuntimeError(
                f"libcco.so not found at {path}; build it with `python xla-cco_b200/build.py` "
                "(there is no CPU fallback)"
            )
        lib = ctypes.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def loaded():
    """The library if an earlier call loaded it, else None (never loads it)."""
    return _lib


class CcoError(RuntimeError):
    """A libcco call failed; ``code`` is the CCO_ERR_* value."""

    def __init__(self, code: int, msg: str) -> None:
        super().__init__(msg)
        self.code = code


def check(code: int, what: str) -> None:
    """Map a CCO return code to the reference's Python exception types."""
    if code == CCO_OK:
        return
    lib = load()
    detail = (lib.cco_last_error() or b"").decode(errors="replace")
    msg = f"{what}: {lib.cco_error_string(code).decode()}" + (f" ({detail})" if detail else "")
    if code == CCO_ERR_ARG:
        raise ValueError(msg)
    raise CcoError(code, msg)


def device_count() -> int:
    """Number of visible CUDA devices (0 when none)."""
    n = ctypes.c_int(0)
    code = load().cco_device_count(ctypes.byref(n))
    return int(n.value) if code == CCO_OK else 0


def require_gpu() -> None:
    """``RuntimeError`` unless a CUDA device is visible (no silent CPU fallback)."""
    if device_count() == 0:
        raise RuntimeError(
            "xla_cco (B200 build) needs a CUDA device: no GPU is visible and there is no CPU path"
        )
