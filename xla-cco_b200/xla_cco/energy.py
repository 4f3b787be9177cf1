"""Stealthy energy in fractional coordinates, evaluated by the sm_100a kernels.

Drop-in for ``xla_cco/energy.py``: ``make_stealthy_energy(box, kset,
chunk_size=None, pad_to=64)`` returns a ``StealthyEnergy`` whose ``__call__``,
``value_and_grad`` and ``value_grad_density`` have the reference's signatures,
error behaviour and results (energy within 1e-12 relative, forces within
1e-12 of max|F| of an exactly reduced FP64 direct sum):

    Phi = (1/V) sum_k w_k |rho_k|^2,   rho_k = sum_j exp(2 pi i n_k . s_j)
    dPhi/ds_j = (2 (2 pi) / V) sum_k w_k (Im rho_k cos th_kj - Re rho_k sin th_kj) n_k

Arrays may be NumPy (results come back as NumPy, host<->device copies
included) or CUDA ``torch`` float64 tensors (results stay on the device).
``chunk_size`` and ``n_max`` are accepted and validated like the reference,
but the kernel tiles itself: no (M, N) matrix is ever formed. Zero rows
(padding) are not sent to the device; their density is exactly (N, 0) and
they carry zero weight.
"""

from __future__ import annotations

import abc
import threading
from typing import Any, Dict, Optional, Tuple

import numpy as np

from xla_cco import _native
from xla_cco._types import require_float64
from xla_cco.box import Box
from xla_cco.kvectors import KSet


def _torch():
    import torch

    return torch


class AbstractEnergy(abc.ABC):
    """Extension point for energies on fractional positions (``energy.py:115-137``).

    A subclass provides ``__call__`` (the scalar energy of one (N, d)
    configuration). As in the reference, ``value_and_grad`` and ``hessian``
    default to automatic differentiation of ``__call__`` - here torch
    autograd, so ``__call__`` must accept a float64 CUDA tensor and use torch
    operations; a subclass may override either with a closed form.
    ``relax`` accepts any subclass: the minimizer lanes run on the device and
    call the energy's ``value_and_grad`` once per tick.
    """

    @abc.abstractmethod
    def __call__(self, s: Any) -> Any:
        """Scalar energy of fractional positions ``s``."""

    def value_and_grad(self, s: Any) -> Tuple[Any, Any]:
        """(energy, dE/ds) by autograd of ``__call__`` (the reference uses
        ``jax.value_and_grad``)."""
        torch = _torch()
        x = _as_cuda(s).detach().clone().requires_grad_(True)
        with torch.enable_grad():
            value = self(x)
            (grad,) = torch.autograd.grad(value, x)
        return value.detach(), grad.detach()

    def hessian(self, s: Any) -> Any:
        """d^2 E / ds ds flattened to (N d, N d), by autograd of ``__call__``
        (the reference uses ``jax.hessian``)."""
        torch = _torch()
        x = _as_cuda(s).detach()
        h = torch.autograd.functional.hessian(lambda y: self(y), x)
        return h.reshape(x.numel(), x.numel())


def _as_cuda(s: Any):
    """``s`` as a float64 CUDA tensor (a NumPy array is copied to the device)."""
    torch = _torch()
    require_float64(s, "s")
    if isinstance(s, torch.Tensor):
        return s if s.is_cuda else s.cuda()
    _native.require_gpu()
    return torch.from_numpy(np.ascontiguousarray(np.asarray(s))).cuda()


class _Problems:
    """Native problem handles of one energy, one per (device, N)."""

    def __init__(self) -> None:
        self._lock = threading.Lock()
        self._handles: Dict[Tuple[int, int], int] = {}

    def get(self, device: int, n_particles: int, n_rows: np.ndarray, w_rows: np.ndarray,
            volume: float) -> int:  # fmt: skip
        key = (device, n_particles)
        with self._lock:
            h = self._handles.get(key)
            if h is not None:
                return h
            lib = _native.load()
            n32 = np.ascontiguousarray(n_rows, dtype=np.int32)
            w64 = np.ascontiguousarray(w_rows, dtype=np.float64)
            out = _native._vp()
            code = lib.cco_problem_create(
                device, int(n32.shape[1]), int(n_particles), int(n32.shape[0]),
                n32.ctypes.data, w64.ctypes.data, float(volume), _native.ctypes.byref(out),
            )  # fmt: skip
            _native.check(code, "cco_problem_create")
            self._handles[key] = int(out.value)
            return self._handles[key]

    def __del__(self) -> None:
        # Handles exist only if the library was loaded to create them; an
        # energy that never reached the device must not map libcco.so here.
        if not self._handles:
            return
        try:   # at interpreter shutdown the module globals may already be gone
            lib = _native.loaded()
            if lib is None:
                return
            for h in self._handles.values():
                lib.cco_problem_destroy(h)
        except Exception:
            pass


class StealthyEnergy(AbstractEnergy):
    """Stealthy energy over a padded k-set (fields as ``energy.py:140-162``).

    n_vectors: (M_pad, d) integer-valued float64, zero rows = padding;
    weights: (M_pad,) float64, 0.0 on padding rows; volume: box volume V;
    chunk_size, n_max: accepted for API compatibility (see module docstring).
    """

    def __init__(self, n_vectors: Any, weights: Any, volume: Any,
                 chunk_size: Optional[int] = None, n_max: Optional[int] = None) -> None:  # fmt: skip
        self.n_vectors = np.asarray(n_vectors)
        self.weights = np.asarray(weights)
        self.volume = np.asarray(volume, dtype=np.float64)
        self.chunk_size = chunk_size
        self.n_max = n_max
        self._check_init()
        a = self.n_vectors
        nz = np.any(a != 0, axis=1)
        self._rows = np.flatnonzero(nz)             # rows sent to the device
        self._zero_rows = np.flatnonzero(~nz)       # padding rows: rho = (N, 0)
        self._zero_weight = float(np.sum(self.weights[~nz])) if a.size else 0.0
        self._n_int = np.rint(a[nz]).astype(np.int64)
        self._w_dev = np.ascontiguousarray(self.weights[nz], dtype=np.float64)
        self._problems = _Problems()

    # ``energy.py:164-184``
    def _check_init(self) -> None:
        a = self.n_vectors
        require_float64(a, "n_vectors")
        if a.ndim != 2:
            raise ValueError("n_vectors must have shape (m, d)")
        if self.n_max is not None and self.n_max < 0:
            raise ValueError(f"n_max must be non-negative, got {self.n_max}")
        if self.n_max is not None and a.size and np.abs(a).max() > self.n_max:
            raise ValueError(f"n_max={self.n_max} is smaller than max|n|={np.abs(a).max():g}")
        if np.any(a != np.round(a)):
            raise ValueError("n_vectors must be integer-valued")
        assert self.chunk_size is None or self.chunk_size >= 1, "chunk_size must be >= 1"

    @property
    def dim(self) -> int:
        return int(self.n_vectors.shape[1])

    # ------------------------------------------------------------ device calls
    def problem_handle(self, device: int, n_particles: int) -> int:
        """Native ``cco_problem*`` for ``n_particles`` on ``device`` (cached)."""
        if self._rows.size == 0:
            raise ValueError("empty k-set: no k-vectors in the shell")
        return self._problems.get(device, n_particles, self._n_int, self._w_dev,
                                  float(self.volume))  # fmt: skip

    def evaluate(self, s: Any, want_grad: bool = True, want_rho: bool = False):
        """Batched evaluation: ``s`` is (B, N, d) float64 (NumPy or CUDA tensor).

        Returns (phi (B,), grad (B,N,d) or None, re (B,M_pad) or None,
        im (B,M_pad) or None) on the same side as the input.
        """
        torch = _torch()
        require_float64(s, "s")
        host = not (isinstance(s, torch.Tensor) and s.is_cuda)
        _native.require_gpu()
        if host:
            st = torch.from_numpy(np.ascontiguousarray(np.asarray(s))).cuda()
        else:
            st = s.contiguous()
        assert st.ndim == 3, "s must have shape (b, n, d)"
        assert st.shape[2] == self.dim, "dimension mismatch"
        b, n, d = st.shape
        dev = st.device.index if st.device.index is not None else torch.cuda.current_device()
        h = self.problem_handle(dev, n)
        m_dev = int(self._rows.size)
        with torch.cuda.device(dev):
            phi = torch.empty(b, dtype=torch.float64, device=st.device)
            grad = torch.empty_like(st) if want_grad else None
            re_d = torch.empty((b, m_dev), dtype=torch.float64, device=st.device) if want_rho else None
            im_d = torch.empty((b, m_dev), dtype=torch.float64, device=st.device) if want_rho else None
            stream = torch.cuda.current_stream(dev).cuda_stream
            code = _native.load().cco_energy_grad(
                h, stream, b, st.data_ptr(), phi.data_ptr(),
                grad.data_ptr() if grad is not None else None,
                re_d.data_ptr() if re_d is not None else None,
                im_d.data_ptr() if im_d is not None else None,
            )  # fmt: skip
            _native.check(code, "cco_energy_grad")
            if self._zero_weight != 0.0:
                phi = phi + self._zero_weight * float(n) * float(n) / float(self.volume)
            re = im = None
            if want_rho:
                mp = self.n_vectors.shape[0]
                re = torch.zeros((b, mp), dtype=torch.float64, device=st.device)
                im = torch.zeros((b, mp), dtype=torch.float64, device=st.device)
                rows = torch.as_tensor(self._rows, device=st.device)
                re[:, rows] = re_d
                im[:, rows] = im_d
                if self._zero_rows.size:
                    re[:, torch.as_tensor(self._zero_rows, device=st.device)] = float(n)
        if host:
            to = lambda t: None if t is None else t.cpu().numpy()  # noqa: E731
            return to(phi), to(grad), to(re), to(im)
        return phi, grad, re, im

    # ------------------------------------------------------------ reference API
    def __call__(self, s: Any) -> Any:
        """Phi(s) for one configuration (N, d) (``energy.py:186-193``)."""
        require_float64(s, "s")
        assert s.ndim == 2, "s must have shape (n, d)"
        assert s.shape[1] == self.dim, "dimension mismatch"
        phi, _, _, _ = self.evaluate(s[None], want_grad=False)
        return float(phi[0]) if isinstance(phi, np.ndarray) else phi[0]

    def value_and_grad(self, s: Any) -> Tuple[Any, Any]:
        """(Phi, dPhi/ds) (``energy.py:195-204``)."""
        value, grad, _, _ = self.value_grad_density(s)
        return value, grad

    def value_grad_density(self, s: Any) -> Tuple[Any, Any, Any, Any]:
        """(Phi, dPhi/ds, Re rho, Im rho) in one pass (``energy.py:206-225``).

        The density covers every row, padding rows included (exactly N, 0).
        """
        require_float64(s, "s")
        assert s.ndim == 2, "s must have shape (n, d)"
        assert s.shape[1] == self.dim, "dimension mismatch"
        phi, grad, re, im = self.evaluate(s[None], want_grad=True, want_rho=True)
        if isinstance(phi, np.ndarray):
            return float(phi[0]), grad[0], re[0], im[0]
        return phi[0], grad[0], re[0], im[0]

    def hessian(self, s: Any) -> Any:
        """Closed-form Hessian d^2 Phi / ds_ja ds_lb flattened to (N d, N d)
        (``energy.py:272-299``), by the ``cco_hessian`` kernels: phases of
        each k-chunk formed in shared memory per particle-tile pair, no
        (N, M) arrays. ``s`` is (N, d), or (B, N, d) for a batch of Hessians
        (B, N d, N d); NumPy in, NumPy out, CUDA tensors stay on the device.
        """
        torch = _torch()
        require_float64(s, "s")
        assert s.ndim in (2, 3), "s must have shape (n, d) or (b, n, d)"
        assert s.shape[-1] == self.dim, "dimension mismatch"
        _native.require_gpu()
        host = not (isinstance(s, torch.Tensor) and s.is_cuda)
        st = torch.from_numpy(np.ascontiguousarray(np.asarray(s))).cuda() if host else s.contiguous()
        batched = st.ndim == 3
        if not batched:
            st = st[None]
        b, n, d = st.shape
        dev = st.device.index if st.device.index is not None else torch.cuda.current_device()
        h = self.problem_handle(dev, n)
        with torch.cuda.device(dev):
            out = torch.empty((b, n * d, n * d), dtype=torch.float64, device=st.device)
            stream = torch.cuda.current_stream(dev).cuda_stream
            for lo in range(0, b, 65535):
                hi = min(b, lo + 65535)
                code = _native.load().cco_hessian(h, stream, hi - lo, st[lo:hi].data_ptr(),
                                                  out[lo:hi].data_ptr())  # fmt: skip
                _native.check(code, "cco_hessian")
        if not batched:
            out = out[0]
        return out.cpu().numpy() if host else out


def auto_chunk_size(n_particles: int, n_vectors: int, budget_bytes: int = 1 << 30,
                    bytes_per_pair: int = 96) -> Optional[int]:  # fmt: skip
    """A ``chunk_size`` whose (c, N) work arrays fit ``budget_bytes``, or None when
    the whole (M, N) matrix fits (``energy.py:86-101``). The device kernels never
    materialise (k, particle) arrays, so ``chunk_size`` is accepted everywhere and
    changes nothing here; this keeps the reference's helper for callers that size
    their own arrays with it."""
    assert n_particles >= 1 and n_vectors >= 1, "sizes must be positive"
    assert budget_bytes >= 1 and bytes_per_pair >= 1, "budget must be positive"
    size = max(1, budget_bytes // (n_particles * bytes_per_pair))
    return None if size >= n_vectors else size


def collective_density(s: Any, n_vectors: Any, chunk_size: Optional[int] = None):
    """(Re rho, Im rho) with rho_k = sum_j exp(2 pi i n_k . s_j) (``energy.py:327-358``)."""
    require_float64(s, "s")
    require_float64(n_vectors, "n_vectors")
    assert s.shape[1] == np.asarray(n_vectors).shape[1], "dimension mismatch"
    assert chunk_size is None or chunk_size >= 1, "chunk_size must be >= 1"
    nv = np.asarray(n_vectors)
    en = _density_energy(nv)
    _, _, re, im = en.evaluate(s[None], want_grad=False, want_rho=True)
    return re[0], im[0]


_DENSITY_CACHE: Dict[bytes, StealthyEnergy] = {}


def _density_energy(nv: np.ndarray) -> StealthyEnergy:
    key = nv.tobytes() + str(nv.shape).encode()
    en = _DENSITY_CACHE.get(key)
    if en is None:
        en = StealthyEnergy(nv, np.ones(nv.shape[0]), np.float64(1.0))
        _DENSITY_CACHE[key] = en
    return en


def make_stealthy_energy(box: Box, kset: KSet, chunk_size: Optional[int] = None,
                         pad_to: int = 64) -> StealthyEnergy:  # fmt: skip
    """Build a ``StealthyEnergy`` from a box and a k-set (``energy.py:361-414``).

    Pads M up to a multiple of ``pad_to`` with zero rows of zero weight;
    ``ValueError`` on an empty k-set.
    """
    require_float64(box.basis, "box.basis")
    assert pad_to >= 1, "pad_to must be >= 1"
    assert chunk_size is None or chunk_size >= 1, "chunk_size must be >= 1"
    m = int(kset.n.shape[0])
    if m == 0:
        raise ValueError("empty k-set: no k-vectors in the shell")
    total = -(-m // pad_to) * pad_to
    n_vec = np.zeros((total, kset.n.shape[1]), dtype=np.float64)
    n_vec[:m] = kset.n
    wts = np.zeros(total, dtype=np.float64)
    wts[:m] = kset.weights
    return StealthyEnergy(n_vec, wts, np.float64(box.volume), chunk_size=chunk_size, n_max=None)
