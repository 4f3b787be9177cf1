"""Structure factor S(k) = |rho(k)|^2 / N and its isotropic average.

Mirrors ``src/xla_cco/analysis/structure.py:44-201`` of the reference (same
names, arguments, outputs and errors). The densities rho(k) come from the
device evaluation kernels (``collective_density`` / ``StealthyEnergy.evaluate``
without the gradient); the k-set construction and the binning are small
host NumPy steps that follow the C++ ``IsotropicStructureFactor`` order
exactly, so the k-set is bit-identical to the reference's.
"""

from __future__ import annotations

import math
from typing import Any, Tuple

import numpy as np

from xla_cco._types import require_float64
from xla_cco.box import Box
from xla_cco.energy import _density_energy, collective_density
from xla_cco.kvectors import enumerate_kvectors

# device scratch per evaluation call: tiles x M partial densities per lane
_SCRATCH_BYTES = 1 << 31


def structure_factor(s: Any, n_vectors: Any) -> Any:
    """S(n) = |rho(n)|^2 / N for integer vectors ``n_vectors`` (M, d)."""
    require_float64(s, "s")
    require_float64(n_vectors, "n_vectors")
    assert s.ndim == 2 and np.asarray(n_vectors).ndim == 2, "expected 2-D arrays"
    re, im = collective_density(s, n_vectors)
    return (re * re + im * im) / s.shape[0]


def isotropic_structure_factor(s: Any, box: Box, k_dir_max: float = 5.0, k_max: float = 400.0,
                               bin_width: float = 0.01) -> Tuple[np.ndarray, ...]:  # fmt: skip
    """Binned isotropic S(|k|) averaged over a batch (b, n, d) of fractional positions.

    One k per primitive direction with |k| < ``k_dir_max`` (half space),
    extended by integer multiples up to |k|^2 <= ``k_max``^2, binned by
    floor(|k| / bin_width). Returns, for every non-empty bin, mean |k|,
    mean S, the standard error of mean |k| (0 unless its variance is
    positive) and the standard error of S (NaN for a negative variance,
    as C++). ``TypeError`` unless float64; ``ValueError`` on bad shapes,
    cutoffs or bin width.
    """
    require_float64(s, "s")
    if s.ndim != 3 or s.shape[2] != box.dim:
        raise ValueError(f"s must have shape (b, n, {box.dim}), got {tuple(s.shape)}")
    if not (0.0 < k_dir_max < k_max and bin_width > 0.0):
        raise ValueError("need 0 < k_dir_max < k_max and bin_width > 0")
    n_vec, k_mod2 = _isotropic_kset(np.asarray(box.basis), k_dir_max, k_max)
    s_mean, s2_mean = _sk_moments(s, n_vec)
    return _bin_moments(np.sqrt(k_mod2), s_mean, s2_mean, int(s.shape[0]), bin_width)


def _isotropic_kset(basis: np.ndarray, k_dir_max: float, k_max: float):
    """Integer vectors (M, d) (float64) and |k|^2 (M,) in the C++ ``GetKs`` order.

    The primitive vectors (coefficient gcd 1) of the half-space shell
    |k| < ``k_dir_max`` in k-set order, each followed by its multiples
    i k, i = 1, 2, ..., while |i k|^2 <= ``k_max``^2 (|i k|^2 summed
    component by component, equality kept). In d = 1 the one direction is
    the reciprocal vector itself, whatever ``k_dir_max``.
    """
    assert basis.ndim == 2 and basis.shape[0] == basis.shape[1], "square basis"
    if basis.shape[0] == 1:
        n_dir = np.ones((1, 1), dtype=np.int64)
        k_dir = np.array([[2.0 * math.pi / basis[0, 0]]])
        q_dir = k_dir[:, 0] ** 2
    else:
        ks = enumerate_kvectors(basis, 0.0, k_dir_max)
        prim = np.gcd.reduce(np.abs(ks.n), axis=1) == 1
        n_dir, k_dir, q_dir = ks.n[prim], ks.k[prim], ks.k_sq[prim]
    if n_dir.shape[0] == 0:
        raise ValueError("no reciprocal-lattice vector below k_dir_max")
    limit = k_max * k_max
    rows, sq = [], []
    for nv, kv, q in zip(n_dir, k_dir, q_dir):
        i = np.arange(1, int(math.sqrt(limit / q)) + 3, dtype=np.float64)
        m2 = np.zeros(i.size)
        for c in range(kv.size):
            comp = i * kv[c]
            m2 = m2 + comp * comp
        keep = m2 <= limit
        rows.append(i[keep, None] * nv[None, :].astype(np.float64))
        sq.append(m2[keep])
    return np.concatenate(rows), np.concatenate(sq)


def _sk_moments(s: Any, n_vec: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Config means of S and S^2 per k (M,), summed over configs in order."""
    import torch

    from xla_cco import _native

    _native.require_gpu()
    b, n = int(s.shape[0]), int(s.shape[1])
    m = int(n_vec.shape[0])
    assert b >= 1 and n >= 1 and m >= 1, "empty input"
    en = _density_energy(np.ascontiguousarray(n_vec))
    st = s if isinstance(s, torch.Tensor) and s.is_cuda else \
        torch.from_numpy(np.ascontiguousarray(np.asarray(s))).cuda()  # fmt: skip
    tiles = -(-n // 64)
    chunk = max(1, min(b, _SCRATCH_BYTES // (16 * m * (tiles + 3))))
    tot = torch.zeros(m, dtype=torch.float64, device=st.device)
    tot2 = torch.zeros_like(tot)
    for lo in range(0, b, chunk):
        _, _, re, im = en.evaluate(st[lo:lo + chunk], want_grad=False, want_rho=True)
        sk = (re * re + im * im) / n
        for row in sk:   # configuration order, as a sequential scan
            tot = tot + row
            tot2 = tot2 + row * row
    return (tot / b).cpu().numpy(), (tot2 / b).cpu().numpy()


def _bin_moments(k_mod: np.ndarray, s_mean: np.ndarray, s2_mean: np.ndarray, n_cfg: int,
                 bin_width: float) -> Tuple[np.ndarray, ...]:  # fmt: skip
    """C++ binning: per bin, sums over k and configurations; empty bins dropped."""
    assert k_mod.shape == s_mean.shape == s2_mean.shape, "shape mismatch"
    idx = np.floor(k_mod / bin_width).astype(np.int64)
    nb = int(idx.max()) + 1
    cnt = np.bincount(idx, minlength=nb) * float(n_cfg)
    nz = cnt != 0
    cnt = cnt[nz]

    def total(v: np.ndarray) -> np.ndarray:
        return np.bincount(idx, weights=v, minlength=nb)[nz] * n_cfg

    mean_k = total(k_mod) / cnt
    mean_s = total(s_mean) / cnt
    var_k = (total(k_mod * k_mod) / cnt - mean_k**2) / cnt
    err_k = np.sqrt(np.where(var_k > 0.0, var_k, 0.0))
    with np.errstate(invalid="ignore"):
        err_s = np.sqrt((total(s2_mean) / cnt - mean_s**2) / cnt)
    return mean_k, mean_s, err_k, err_s
