"""Observables of the tracked waves (``src/xla_cco/dynamics/observables.py:56-125``).

``wave_densities`` sums on the GPU (torch, FP64); the others are O(w)
bookkeeping on the caller's arrays. Inside ``simulate`` all of them run in
the MD tick on the device (``cco_md_segment``); these are the same
definitions for analysis and for single steps.
"""

from __future__ import annotations

from typing import Any, Optional, Tuple

import numpy as np

from xla_cco import _native
from xla_cco._types import require_float64


def wave_densities(r: Any, kvec: Any, chunk_size: Optional[int] = None) -> Any:
    """rho_k = sum_j exp(i k . r_j) as (w, 2) (Re, Im) at Cartesian r (n, d)."""
    import torch

    require_float64(r, "r")
    require_float64(kvec, "kvec")
    assert r.ndim == 2 and kvec.ndim == 2 and r.shape[1] == kvec.shape[1], "shapes"
    assert chunk_size is None or chunk_size >= 1, "chunk_size must be >= 1"
    _native.require_gpu()
    host = not (isinstance(r, torch.Tensor) and r.is_cuda)
    rt = torch.as_tensor(np.asarray(r) if host else r, dtype=torch.float64).cuda()
    kt = torch.as_tensor(np.asarray(kvec) if not isinstance(kvec, torch.Tensor) else kvec,
                         dtype=torch.float64).to(rt.device)  # fmt: skip
    step = kt.shape[0] if chunk_size is None else int(chunk_size)
    rows = []
    for lo in range(0, kt.shape[0], step):
        th = kt[lo:lo + step] @ rt.T
        rows.append(torch.stack([torch.cos(th).sum(1), torch.sin(th).sum(1)], -1))
    out = torch.cat(rows) if rows else torch.zeros((0, 2), dtype=torch.float64, device=rt.device)
    return out.cpu().numpy() if host else out


def center_of_mass(r: np.ndarray) -> np.ndarray:
    """Mean position (mass 1, unwrapped coordinates)."""
    require_float64(r, "r")
    assert r.ndim == 2 and r.shape[0] >= 1, "r must have shape (n, d)"
    return np.mean(r, axis=0)


def com_correct(rho: np.ndarray, kvec: np.ndarray, r_cm: np.ndarray) -> np.ndarray:
    """rho_k exp(-i k . R_cm): translation-invariant densities."""
    assert rho.ndim == 2 and rho.shape[1] == 2 and kvec.shape == (rho.shape[0], r_cm.shape[0])
    ph = kvec @ r_cm
    c, s = np.cos(ph), np.sin(ph)
    re, im = rho[:, 0], rho[:, 1]
    return np.stack([re * c + im * s, im * c - re * s], axis=-1)


def winding_update(rho_prev: np.ndarray, rho_new: np.ndarray, wind_abs: np.ndarray,
                   wind_net: np.ndarray, n_valid: np.ndarray, active: np.ndarray, n_part: int,
                   phase_floor: float) -> Tuple[np.ndarray, ...]:  # fmt: skip
    """(rho_prev', wind_abs', wind_net', n_valid'): the step's phase change
    atan2(Im p, Re p), p = rho_new conj(rho_old), counts where the wave is
    ``active`` and S = |rho|^2 / n_part exceeds ``phase_floor`` at both ends."""
    assert n_part >= 1, "n_part must be positive"
    o_re, o_im = rho_prev[:, 0], rho_prev[:, 1]
    n_re, n_im = rho_new[:, 0], rho_new[:, 1]
    delta = np.arctan2(n_im * o_re - n_re * o_im, n_re * o_re + n_im * o_im)
    s_old = (o_re * o_re + o_im * o_im) / n_part
    s_new = (n_re * n_re + n_im * n_im) / n_part
    ok = active & (s_old > phase_floor) & (s_new > phase_floor)
    return (np.where(active[:, None], rho_new, rho_prev), wind_abs + np.where(ok, np.abs(delta), 0.0),
            wind_net + np.where(ok, delta, 0.0), n_valid + ok.astype(n_valid.dtype))  # fmt: skip
