"""TEST INFRASTRUCTURE ONLY: the CPU oracle (checker) for the hot path.

Imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg only - never by the product (``xla-cco_b200/xla_cco``), which has no CPU
path. Wraps ``cco_oracle.c`` (built by ``oracle/build.py`` into
``oracle/liboracle.so``) and adds small pure-Python restatements:

* ``halfspace_kvectors``: brute-force k scan (``tests/oracle.py:114-150`` of
  the reference), independent of the product's vectorized enumeration;
* ``energy_direct``: NumPy direct sum of the trig path
  (``src/xla_cco/energy.py:45-50,301-324``), for small cases.

Parity pins (tests/golden/, generated from the reference by
``tests/golden/make_golden.py``): C++ golden energies of
``tests/data/md_cxx_samples.npz``, the reference oracle's energies and
forces, the reference k-set enumeration, and the reference test's verbatim
transcription of the C++ descent loop. L-BFGS iterates are unpinned (optax
is not vendored); its statuses and accounting are checked behaviourally.
"""

from __future__ import annotations

import ctypes
import itertools
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SRC = HERE / "cco_oracle.c"


def build(force: bool = False) -> Path:
    """Compile liboracle.so with gcc (OpenMP) if missing or stale."""
    if force or not LIB.exists() or SRC.stat().st_mtime > LIB.stat().st_mtime:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=gnu11", "-o", str(tmp),
               str(SRC), "-lm"]  # fmt: skip
        subprocess.run(cmd, check=True)
        tmp.replace(LIB)
    return LIB


_lib = None


class DescentC(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("step_init", "step_min", "shrink", "grow", "rel_tol")] + [
        ("max_evals", ctypes.c_int64),
        ("energy_tol", ctypes.c_double),
        ("record_every", ctypes.c_int64),
        ("max_records", ctypes.c_int64),
    ]


class LBFGSC(ctypes.Structure):
    _fields_ = [
        ("memory", ctypes.c_int64),
        ("n_rescales", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("rescales", ctypes.c_double * 8),
        ("max_evals_per_pass", ctypes.c_int64),
        ("energy_tol", ctypes.c_double),
        ("grad_tol", ctypes.c_double),
        ("stagnation_patience", ctypes.c_int64),
        ("max_linesearch_steps", ctypes.c_int64),
        ("record_every", ctypes.c_int64),
        ("max_records", ctypes.c_int64),
    ]


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(build()))
        _lib.oracle_energy_grad.restype = ctypes.c_double
        _lib.oracle_max_threads.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def energy_grad(s: np.ndarray, n: np.ndarray, w: np.ndarray, volume: float,
                want_rho: bool = False):  # fmt: skip
    """(Phi, dPhi/ds[, re, im]) of one configuration by the C direct sum."""
    s = np.ascontiguousarray(s, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    N, d = s.shape
    M = n.shape[0]
    g = np.zeros_like(s)
    re = np.zeros(M) if want_rho else None
    im = np.zeros(M) if want_rho else None
    phi = lib().oracle_energy_grad(
        ctypes.c_int(N), ctypes.c_int(d), _p(s), ctypes.c_int(M), _p(n), _p(w),
        ctypes.c_double(volume), _p(g), _p(re), _p(im),
    )  # fmt: skip
    return (phi, g, re, im) if want_rho else (phi, g)


def energy_grad_batch(s: np.ndarray, n: np.ndarray, w: np.ndarray, volume: float,
                      threads: int = 0):  # fmt: skip
    """Batched (B, N, d) energies and gradients, OpenMP over configurations."""
    s = np.ascontiguousarray(s, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    B, N, d = s.shape
    phi = np.zeros(B)
    g = np.zeros_like(s)
    lib().oracle_energy_grad_batch(
        ctypes.c_int(B), ctypes.c_int(N), ctypes.c_int(d), _p(s), ctypes.c_int(n.shape[0]),
        _p(n), _p(w), ctypes.c_double(volume), _p(phi), _p(g), ctypes.c_int(threads),
    )  # fmt: skip
    return phi, g


def _descent_c(st) -> DescentC:
    return DescentC(st.step_init, st.step_min, st.shrink, st.grow, st.rel_tol, st.max_evals,
                    st.energy_tol, st.record_every, st.max_records)  # fmt: skip


def _lbfgs_c(st) -> LBFGSC:
    c = LBFGSC()
    c.memory = st.memory
    c.n_rescales = len(st.rescales)
    for i, r in enumerate(st.rescales):
        c.rescales[i] = r
    c.max_evals_per_pass = st.max_evals_per_pass
    c.energy_tol = st.energy_tol
    c.grad_tol = st.grad_tol
    c.stagnation_patience = st.stagnation_patience
    c.max_linesearch_steps = st.max_linesearch_steps
    c.record_every = st.record_every
    c.max_records = st.max_records
    return c


def relax_one(method: str, s0: np.ndarray, n: np.ndarray, w: np.ndarray, volume: float,
              settings) -> dict:  # fmt: skip
    """One relaxation ('descent' or 'lbfgs') with the trajectory when recording."""
    s0 = np.ascontiguousarray(s0, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    N, d = s0.shape
    nd = N * d
    cap = settings.max_records if (settings.record_every > 0 and settings.max_records > 0) else 0
    out = dict(s=np.zeros_like(s0), energy=np.zeros(1), grad_norm=np.zeros(1),
               n_evals=np.zeros(1, np.int64), n_iters=np.zeros(1, np.int64),
               status=np.zeros(1, np.int64))  # fmt: skip
    ts = np.zeros((max(cap, 1), N, d))
    te, tst = np.zeros(max(cap, 1)), np.zeros(max(cap, 1))
    tit = np.zeros(max(cap, 1), np.int64)
    tc = np.zeros(1, np.int64)
    if method == "descent":
        c, fn = _descent_c(settings), lib().oracle_descent
    else:
        c, fn = _lbfgs_c(settings), lib().oracle_lbfgs
    rec = cap > 0
    fn(ctypes.c_int(N), ctypes.c_int(d), _p(s0), ctypes.c_int(n.shape[0]), _p(n), _p(w),
       ctypes.c_double(volume), ctypes.byref(c), _p(out["s"]), _p(out["energy"]),
       _p(out["grad_norm"]), _p(out["n_evals"]), _p(out["n_iters"]), _p(out["status"]),
       _p(ts) if rec else None, _p(te) if rec else None, _p(tst) if rec else None,
       _p(tit) if rec else None, _p(tc) if rec else None)  # fmt: skip
    res = {k: (v if k == "s" else v[0]) for k, v in out.items()}
    if rec:
        res["trajectory"] = dict(s=ts, energy=te, step=tst, iteration=tit, count=int(tc[0]))
    del nd
    return res


def relax_batch(method: str, s0: np.ndarray, n: np.ndarray, w: np.ndarray, volume: float,
                settings, threads: int = 0) -> dict:  # fmt: skip
    """Batched relaxations (OpenMP over lanes); lanes are independent."""
    s0 = np.ascontiguousarray(s0, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    B, N, d = s0.shape
    out = dict(s=np.zeros_like(s0), energy=np.zeros(B), grad_norm=np.zeros(B),
               n_evals=np.zeros(B, np.int64), n_iters=np.zeros(B, np.int64),
               status=np.zeros(B, np.int64))  # fmt: skip
    c = _descent_c(settings) if method == "descent" else _lbfgs_c(settings)
    lib().oracle_relax_batch(
        ctypes.c_int(0 if method == "descent" else 1), ctypes.c_int(B), ctypes.c_int(N),
        ctypes.c_int(d), _p(s0), ctypes.c_int(n.shape[0]), _p(n), _p(w), ctypes.c_double(volume),
        ctypes.byref(c), _p(out["s"]), _p(out["energy"]), _p(out["grad_norm"]),
        _p(out["n_evals"]), _p(out["n_iters"]), _p(out["status"]), ctypes.c_int(threads),
    )  # fmt: skip
    return out


def max_threads() -> int:
    return int(lib().oracle_max_threads())


# ------------------------------------------------------------ pure Python


def reciprocal_basis(basis: np.ndarray) -> np.ndarray:
    return 2.0 * math.pi * np.linalg.inv(basis).T


def modulus2(k: np.ndarray) -> float:
    """|k|^2 summed component by component in index order (C++ Modulus2)."""
    acc = 0.0
    for c in range(k.shape[0]):
        acc += float(k[c]) * float(k[c])
    return acc


def halfspace_kvectors(basis: np.ndarray, k_inner: float, k_outer: float):
    """Brute-force half-space scan with strict K1^2 < |k|^2 < K2^2 (small cases)."""
    dim = basis.shape[0]
    recip = reciprocal_basis(basis)
    bounds = [int(math.floor(k_outer * float(np.linalg.norm(basis[i])) / (2.0 * math.pi))) + 1
              for i in range(dim)]  # fmt: skip
    found, ksq = [], []
    for nn in itertools.product(*[range(-b, b + 1) for b in bounds]):
        nz = [c for c in nn if c != 0]
        if not nz or nz[0] < 0:
            continue
        k = np.array(nn, dtype=np.float64) @ recip
        q = modulus2(k)
        if k_inner * k_inner < q < k_outer * k_outer:
            found.append(nn)
            ksq.append(q)
    return np.array(found, dtype=np.int64).reshape(-1, dim), np.array(ksq)


def energy_direct(s: np.ndarray, n: np.ndarray, w: np.ndarray, volume: float):
    """NumPy direct sum (Phi, dPhi/ds) of the trig path (small N * M)."""
    theta = 2.0 * math.pi * (n.astype(np.float64) @ s.T)  # (M, N)
    c, si = np.cos(theta), np.sin(theta)
    re, im = c.sum(1), si.sum(1)
    phi = float(np.sum(w * (re * re + im * im)) / volume)
    coef = w[:, None] * (im[:, None] * c - re[:, None] * si)  # (M, N)
    grad = (2.0 * 2.0 * math.pi / volume) * (coef.T @ n.astype(np.float64))
    return phi, grad
