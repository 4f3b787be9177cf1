"""Pair statistics: nearest-neighbour distances, pair histograms and g2.

Mirrors ``src/xla_cco/analysis/pairs.py:41-136`` of the reference (same
names, arguments, outputs and errors). Distances are minimum-image in
length units (ds - round(ds), then the 3^d image shifts through the
basis): positions must be wrapped to [0, 1) and the cell reduced, as in
the reference. The O(N^2) work runs in the ``cco_pair_histogram`` and
``cco_nearest_neighbor`` kernels; counts are exact integers.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from xla_cco import _native
from xla_cco._types import require_float64
from xla_cco.box import Box
from xla_cco.kvectors import unit_ball_volume


def _device_positions(s: Any):
    import torch

    _native.require_gpu()
    if isinstance(s, torch.Tensor) and s.is_cuda:
        return s.contiguous(), False
    return torch.from_numpy(np.ascontiguousarray(np.asarray(s))).cuda(), True


def _basis(box: Box) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(box.basis, dtype=np.float64))


def nearest_neighbor_distances(s: Any, box: Box) -> Any:
    """Minimum-image nearest-neighbour distance of every particle of (n, d) ``s``.

    A lone particle sees its own nearest periodic image. ``TypeError``
    unless float64.
    """
    import torch

    require_float64(s, "s")
    assert s.ndim == 2 and s.shape[1] == box.dim, "s must have shape (n, d)"
    st, host = _device_positions(s)
    n, d = st.shape
    basis = _basis(box)
    dev = st.device.index if st.device.index is not None else torch.cuda.current_device()
    with torch.cuda.device(dev):
        out = torch.empty(n, dtype=torch.float64, device=st.device)
        stream = torch.cuda.current_stream(dev).cuda_stream
        code = _native.load().cco_nearest_neighbor(
            dev, stream, 1, n, d, st.data_ptr(), basis.ctypes.data, out.data_ptr())
        _native.check(code, "cco_nearest_neighbor")
    return out.cpu().numpy() if host else out


def nearest_neighbor_distances_batch(s: Any, box: Box) -> Any:
    """Nearest-neighbour distances (b, n) of a batch (b, n, d) in one kernel
    call per 65535 configurations (no reference counterpart: the reference
    maps ``nearest_neighbor_distances`` over configurations). A CUDA input
    gives a CUDA result; NumPy in, NumPy out."""
    import torch

    require_float64(s, "s")
    assert s.ndim == 3 and s.shape[2] == box.dim, "s must have shape (b, n, d)"
    st, host = _device_positions(s)
    b, n, d = st.shape
    basis = _basis(box)
    dev = st.device.index if st.device.index is not None else torch.cuda.current_device()
    with torch.cuda.device(dev):
        out = torch.empty((b, n), dtype=torch.float64, device=st.device)
        stream = torch.cuda.current_stream(dev).cuda_stream
        for lo in range(0, b, 65535):
            hi = min(b, lo + 65535)
            code = _native.load().cco_nearest_neighbor(
                dev, stream, hi - lo, n, d, st[lo:hi].data_ptr(), basis.ctypes.data,
                out[lo:hi].data_ptr())  # fmt: skip
            _native.check(code, "cco_nearest_neighbor")
    return out.cpu().numpy() if host else out


def pair_distance_histogram(s: Any, box: Box, edges: np.ndarray) -> np.ndarray:
    """int64 pair counts (every i < j once per configuration) of (b, n, d) ``s``.

    Bins follow ``np.histogram`` ([e_k, e_k+1), the last one closed);
    distances outside [edges[0], edges[-1]] are not counted. ``TypeError``
    unless float64; ``ValueError`` unless ``edges`` is 1-D, finite,
    non-negative and strictly increasing.
    """
    import torch

    require_float64(s, "s")
    _check_edges(edges)
    assert s.ndim == 3 and s.shape[2] == box.dim, "s must have shape (b, n, d)"
    st, _ = _device_positions(s)
    b, n, d = st.shape
    e = np.ascontiguousarray(np.asarray(edges, dtype=np.float64))
    basis = _basis(box)
    dev = st.device.index if st.device.index is not None else torch.cuda.current_device()
    with torch.cuda.device(dev):
        counts = torch.empty(e.size - 1, dtype=torch.int64, device=st.device)
        stream = torch.cuda.current_stream(dev).cuda_stream
        for lo in range(0, b, 65535):
            part = torch.empty_like(counts) if lo else counts
            hi = min(b, lo + 65535)
            code = _native.load().cco_pair_histogram(
                dev, stream, hi - lo, n, d, st[lo:hi].data_ptr(), basis.ctypes.data, int(e.size),
                e.ctypes.data, part.data_ptr())  # fmt: skip
            _native.check(code, "cco_pair_histogram")
            if lo:
                counts += part
    return counts.cpu().numpy()


def g2_from_histogram(counts: np.ndarray, edges: np.ndarray, n_particles: int, n_configs: int,
                      volume: float, dim: int) -> np.ndarray:  # fmt: skip
    """g2 = counts / [(V_d r_hi^d - V_d r_lo^d) * 0.5 * rho * N * n_configs], rho = N / V.

    Pairs are counted once (the C++ ``PairCorrelation`` normalisation).
    """
    _check_edges(edges)
    edges = np.asarray(edges, dtype=np.float64)
    if np.asarray(counts).shape != (edges.shape[0] - 1,):
        raise ValueError("counts must have length len(edges) - 1")
    assert n_particles >= 1 and n_configs >= 1 and dim >= 1, "bad sizes"
    assert volume > 0.0, "volume must be positive"
    vd = unit_ball_volume(dim)
    shell = vd * edges[1:] ** dim - vd * edges[:-1] ** dim
    rho = n_particles / volume
    return np.asarray(counts, dtype=np.float64) / (shell * 0.5 * rho * n_particles * n_configs)


def _check_edges(edges: Any) -> None:
    e = np.asarray(edges)
    if e.ndim != 1 or e.shape[0] < 2:
        raise ValueError("edges must be 1-D with at least 2 entries")
    if not np.all(np.isfinite(e)) or e[0] < 0.0:
        raise ValueError("edges must be finite and non-negative")
    if not np.all(np.diff(e) > 0.0):
        raise ValueError("edges must be strictly increasing")
