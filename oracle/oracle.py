"""TEST INFRASTRUCTURE ONLY: the CPU oracle (checker) for the hot path.

Imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg only - never by the product (``xla-cco_b200/xla_cco``), which has no CPU
path. Wraps ``cco_oracle.c`` (built by ``oracle/build.py`` into
``oracle/liboracle.so``) and adds small pure-Python restatements:

* ``halfspace_kvectors``: brute-force k scan (``tests/oracle.py:114-150`` of
  the reference), independent of the product's vectorized enumeration;
* ``energy_direct``: NumPy direct sum of the trig path
  (``src/xla_cco/energy.py:45-50,301-324``), for small cases;
* ``structure_factor_direct``, ``isotropic_kset``, ``bin_moments``: S(k)
  by direct sums, the C++ ``GetKs`` k-set by brute force and the C++ S(k)
  binning in plain Python (``src/xla_cco/analysis/structure.py:44-201``);
* ``min_image_distances``: minimum-image pair and nearest-neighbour
  distances (``src/xla_cco/analysis/pairs.py:41-188``).

Parity pins (tests/golden/io_golden.*, generated from the reference by
``tests/golden/make_io_golden.py``): the reference's own ``_isotropic_kset``
and ``_bin_moments`` outputs, its oracle's pair distances and S(k), and its
ConfigPack and table writers' bytes.

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


def lbfgs_settings(**overrides):
    """Settings object with the reference's LBFGSSettings fields and defaults
    (src/xla_cco/minimize/lbfgs.py:55-67), for callers that must not import
    the product package."""
    import types

    base = dict(memory=100, rescales=(1e4, 1.0, 1e-2), max_evals_per_pass=500_000,
                energy_tol=0.0, grad_tol=0.0, stagnation_patience=50, max_linesearch_steps=30,
                record_every=0, max_records=0)  # fmt: skip
    base.update(overrides)
    return types.SimpleNamespace(**base)


def energy_grad_accurate(s: np.ndarray, n: np.ndarray, w: np.ndarray, volume: float,
                         want_rho: bool = False, threads: int = 0):  # fmt: skip
    """(Phi, dPhi/ds[, re, im]) of a batch (B, N, d) with the phase argument
    reduced exactly and compensated sums (cco_oracle.c): a higher-accuracy
    reference than the FP64 trig path, for measuring the kernels' own error."""
    s = np.ascontiguousarray(s, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    B, N, d = s.shape
    M = n.shape[0]
    phi, g = np.zeros(B), np.zeros_like(s)
    re = np.zeros((B, M)) if want_rho else None
    im = np.zeros((B, M)) if want_rho else None
    lib().oracle_energy_grad_accurate_batch(
        ctypes.c_int(B), ctypes.c_int(N), ctypes.c_int(d), _p(s), ctypes.c_int(M), _p(n), _p(w),
        ctypes.c_double(volume), _p(phi), _p(g), _p(re), _p(im),
        ctypes.c_int(threads or max_threads()),
    )  # fmt: skip
    return (phi, g, re, im) if want_rho else (phi, g)


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


def relax_lanes(method: str, s0: np.ndarray, n: np.ndarray, w: np.ndarray, volume: float,
                settings, threads: int = 0) -> dict:  # fmt: skip
    """The lanes of ``relax_batch`` one after another, each evaluation spread
    over ``threads`` host threads (same bits as ``relax_batch``)."""
    s0 = np.ascontiguousarray(s0, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    B, N, d = s0.shape
    out = dict(s=np.zeros_like(s0), energy=np.zeros(B), grad_norm=np.zeros(B),
               n_evals=np.zeros(B, np.int64), n_iters=np.zeros(B, np.int64),
               status=np.zeros(B, np.int64))  # fmt: skip
    c = _descent_c(settings) if method == "descent" else _lbfgs_c(settings)
    lib().oracle_relax_lanes(
        ctypes.c_int(0 if method == "descent" else 1), ctypes.c_int(B), ctypes.c_int(N),
        ctypes.c_int(d), _p(s0), ctypes.c_int(n.shape[0]), _p(n), _p(w), ctypes.c_double(volume),
        ctypes.byref(c), _p(out["s"]), _p(out["energy"]), _p(out["grad_norm"]),
        _p(out["n_evals"]), _p(out["n_iters"]), _p(out["status"]),
        ctypes.c_int(threads or max_threads()),
    )  # fmt: skip
    return out


def max_threads() -> int:
    return int(lib().oracle_max_threads())


# ------------------------------------------------------------ cutoffs and k-sets
# Unit-ball volumes for d <= 3 as the C++ engine hard-codes them
# (src/xla_cco/kvectors.py:131-149 keeps those literals).
_UNIT_BALL = {1: 2.0, 2: math.pi, 3: 4.1887902047863909846}


def k_outer_for_chi(chi: float, phi: float, dim: int) -> float:
    """K2 for a target chi (src/xla_cco/kvectors.py:152-163 restated):
    Ka = (2^(d+1) d chi Gamma(d/2+1)^2 phi)^(1/d), a = (phi / V_d)^(1/d), K2 = Ka / a."""
    ka = (2.0 ** (dim + 1) * dim * chi * math.gamma(dim / 2.0 + 1.0) ** 2 * phi) ** (1.0 / dim)
    a = (phi / _UNIT_BALL[dim]) ** (1.0 / dim)
    return ka / a


def sorted_kset(basis: np.ndarray, k_inner: float, k_outer: float) -> np.ndarray:
    """The brute-force half-space scan ordered as the reference orders its
    k-set (src/xla_cco/kvectors.py:91-93): by |k|^2, then n_0, n_1, ..."""
    n, ksq = halfspace_kvectors(basis, k_inner, k_outer)
    keys = tuple(n[:, i] for i in range(n.shape[1] - 1, -1, -1)) + (ksq,)
    return n[np.lexsort(keys)]


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


def hessian_direct(s: np.ndarray, n: np.ndarray, w: np.ndarray, volume: float) -> np.ndarray:
    """Closed-form Hessian (N d, N d) of one configuration by NumPy direct sums
    (src/xla_cco/energy.py:272-299 restated):
    d2 Phi / ds_ja ds_lb = (2 (2 pi)^2 / V) sum_k w_k n_ka n_kb
    [cos th_kj cos th_kl + sin th_kj sin th_kl - delta_jl (Re rho_k cos th_kj + Im rho_k sin th_kj)].
    Small cases only (forms (N, M) matrices)."""
    nf = np.asarray(n, dtype=np.float64)
    N, d = s.shape
    theta = 2.0 * math.pi * (s @ nf.T)          # (N, M)
    c, si = np.cos(theta), np.sin(theta)
    re, im = c.sum(0), si.sum(0)
    pref = 2.0 * (2.0 * math.pi) ** 2 / volume
    out = np.zeros((N, d, N, d))
    for a in range(d):
        for b in range(d):
            q = w * nf[:, a] * nf[:, b]
            pair = (c * q) @ c.T + (si * q) @ si.T
            out[:, a, :, b] = pref * (pair - np.diag((re * c + im * si) @ q))
    return out.reshape(N * d, N * d)


# ------------------------------------------------------------------ gradient flow
# Dormand & Prince (1980) 5(4) tableau, the published coefficients.
_DP_A = (
    (),
    (1 / 5,),
    (3 / 40, 9 / 40),
    (44 / 45, -56 / 15, 32 / 9),
    (19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729),
    (9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656),
)
_DP_B5 = (35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0.0)
_DP_B4 = (5179 / 57600, 0.0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40)
_DP_E = tuple(b5 - b4 for b5, b4 in zip(_DP_B5, _DP_B4))


def gradient_flow_dopri5(s0: np.ndarray, n: np.ndarray, w: np.ndarray, volume: float,
                         basis: np.ndarray, st, dt0: float | None = None) -> dict:  # fmt: skip
    """Restatement of the reference's DoPri5 gradient flow for one lane
    (``src/xla_cco/minimize/flow.py:258-364,401-451``), energies and gradients
    from the C direct sum. ``st`` carries the FlowSettings fields. Returns the
    final state and, when recording, the trajectory rows."""
    basis = np.asarray(basis, dtype=np.float64)
    metric_inv = np.linalg.inv(basis @ basis.T)
    binv_t = np.linalg.inv(basis).T
    arc = st.parametrization == "arclength"

    def velocity(s):
        f, g = energy_grad(s, n, w, volume)
        v = -g @ metric_inv
        gn = float(np.sqrt(np.sum((g @ binv_t) ** 2)))
        if not arc:
            return f, g, v, np.array([1.0, gn]), gn
        inv = 1.0 / gn if gn > 0.0 else 0.0
        return f, g, v * inv, np.array([inv, 1.0]), gn

    def status(f, g, gn, t, dt, steps, tries):
        code = 2 if dt < st.dt_min else 0
        if t >= st.t_max or steps >= st.max_steps or tries >= 4 * st.max_steps:
            code = 3
        if np.all(g == 0.0) or gn < st.grad_tol:
            code = 6
        return 1 if f < st.energy_tol else code

    s = np.array(s0, dtype=np.float64)
    f, g, v, rate, gn = velocity(s)
    dt = min(st.dt_init if dt0 is None else dt0, st.dt_max)
    t = length = 0.0
    steps = tries = 0
    evals = 1
    rows = [(s.copy(), 0.0, 0.0, f)]
    code = status(f, g, gn, 0.0, dt, 0, 0)
    while code == 0:
        h = dt if arc else min(dt, st.t_max - t)
        ks, rates = [v], [rate]
        for i in range(1, 6):
            incr = sum(a * k for a, k in zip(_DP_A[i], ks))
            _, _, vi, ri, _ = velocity(s + h * incr)
            ks.append(vi)
            rates.append(ri)
        s_new = s + h * sum(b * k for b, k in zip(_DP_B5[:6], ks))
        tl = h * sum(b * r for b, r in zip(_DP_B5[:6], rates))
        f_new, g_new, v_new, r_new, gn_new = velocity(s_new)
        err_s = h * sum(e * k for e, k in zip(_DP_E, ks + [v_new]))
        err_tl = h * sum(e * r for e, r in zip(_DP_E, rates + [r_new]))
        move = np.sqrt(np.mean(((s_new - s) @ basis) ** 2))
        err = np.sqrt(np.mean((err_s @ basis) ** 2)) / (st.atol + st.rtol * move)
        err = max(err, float(np.max(np.abs(err_tl) / (st.atol + st.rtol * np.abs(tl)))))
        accept = err <= 1.0
        with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
            factor = float(np.clip(0.9 * err ** (-1.0 / 5.0), 0.2, 5.0))
        if not math.isfinite(factor):
            factor = 0.2
        dt = min(h * factor, st.dt_max)
        if accept:
            s, f, g, v, rate, gn = s_new, f_new, g_new, v_new, r_new, gn_new
            t += tl[0]
            length += tl[1]
            steps += 1
        tries += 1
        evals += 6
        code = status(f, g, gn, t, dt, steps, tries)
        if (accept and st.record_every > 0 and steps % st.record_every == 0
                and len(rows) < st.max_records):  # fmt: skip
            rows.append((s.copy(), t, length, f))
    out = dict(s=s, energy=f, t=t, length=length, dt=dt, n_steps=steps, n_evals=evals,
               status=code)  # fmt: skip
    if st.record_every > 0:
        if not (rows[-1][2] == length and rows[-1][1] == t):
            if len(rows) >= st.max_records:
                rows[-1] = (s.copy(), t, length, f)
            else:
                rows.append((s.copy(), t, length, f))
        out["trajectory"] = rows
    return out


# ------------------------------------------------------------------ analysis


def structure_factor_direct(s: np.ndarray, n: np.ndarray) -> np.ndarray:
    """S(n) = |sum_j exp(2 pi i n . s_j)|^2 / N by direct NumPy sums (small cases)."""
    theta = 2.0 * math.pi * (np.asarray(n, dtype=np.float64) @ s.T)
    re, im = np.cos(theta).sum(1), np.sin(theta).sum(1)
    return (re * re + im * im) / s.shape[0]


def isotropic_kset(basis: np.ndarray, k_dir: float, k_max: float):
    """C++ ``GetKs`` by brute force: primitive half-space vectors with |k| < k_dir
    ordered by (|k|^2, n_0, n_1, ...), each followed by its multiples i n while
    |i k|^2 <= k_max^2 (summed component by component). d = 1: the one
    direction n = 1 whatever k_dir."""
    dim = basis.shape[0]
    recip = reciprocal_basis(basis)
    if dim == 1:
        prim = [np.array([1], dtype=np.int64)]
    else:
        found, ksq = halfspace_kvectors(basis, 0.0, k_dir)
        order = sorted(range(len(ksq)), key=lambda i: (ksq[i], tuple(found[i])))
        prim = []
        for i in order:
            g = 0
            for c in found[i]:
                g = math.gcd(g, abs(int(c)))
            if g == 1:
                prim.append(found[i])
    rows, sq = [], []
    for nv in prim:
        kv = nv.astype(np.float64) @ recip if dim > 1 else np.array([recip[0, 0]])
        i = 1
        while True:
            q = 0.0
            for c in range(dim):
                comp = float(i) * float(kv[c])
                q += comp * comp
            if q > k_max * k_max:
                break
            rows.append([float(i) * float(x) for x in nv])
            sq.append(q)
            i += 1
    return np.array(rows, dtype=np.float64), np.array(sq, dtype=np.float64)


def bin_moments(k: np.ndarray, s_mean: np.ndarray, s2_mean: np.ndarray, n_cfg: int,
                width: float):
    """C++ S(k) binning in plain Python: per bin floor(|k| / width), totals over k
    and configurations, mean |k|, mean S, SEM of |k| (0 unless the variance is
    positive) and SEM of S (NaN for a negative variance)."""
    acc: dict[int, list[float]] = {}
    for kk, sm, s2 in zip(k.tolist(), s_mean.tolist(), s2_mean.tolist()):
        b = int(math.floor(kk / width))
        a = acc.setdefault(b, [0.0, 0.0, 0.0, 0.0, 0.0])
        a[0] += 1.0
        a[1] += kk
        a[2] += sm
        a[3] += kk * kk
        a[4] += s2
    cols: list[list[float]] = [[], [], [], []]
    for b in sorted(acc):
        a = acc[b]
        cnt = a[0] * float(n_cfg)
        mk, ms = a[1] * n_cfg / cnt, a[2] * n_cfg / cnt
        vk = (a[3] * n_cfg / cnt - mk * mk) / cnt
        vs = (a[4] * n_cfg / cnt - ms * ms) / cnt
        cols[0].append(mk)
        cols[1].append(ms)
        cols[2].append(math.sqrt(vk) if vk > 0.0 else 0.0)
        cols[3].append(math.sqrt(vs) if vs >= 0.0 else math.nan)
    return tuple(np.array(c) for c in cols)


def min_image_distances(s: np.ndarray, basis: np.ndarray):
    """(nearest-neighbour distance per particle (N,), distances of pairs i < j
    in row order) with ds - round(ds) and the 3^d image shifts; a particle's
    own zero shift is excluded (a lone particle sees its images)."""
    n, dim = s.shape
    shifts = np.array(list(itertools.product((-1.0, 0.0, 1.0), repeat=dim)))
    ds = s[None, :, :] - s[:, None, :]
    ds = ds - np.round(ds)
    best = np.full((n, n), np.inf)
    for sh in shifts:
        v = (ds + sh) @ basis
        r2 = (v * v).sum(-1)
        if not sh.any():
            r2 = np.where(np.eye(n, dtype=bool), np.inf, r2)
        best = np.minimum(best, r2)
    dist = np.sqrt(best)
    iu = np.triu_indices(n, 1)
    return dist.min(axis=1), dist[iu]


# ------------------------------------------------------------------ MD observables
# Restates src/xla_cco/dynamics/observables.py:56-125 and the per-step
# bookkeeping of src/xla_cco/dynamics/run.py:247-280,415-496 in NumPy.


def density_direct(s: np.ndarray, n: np.ndarray):
    """(Re rho, Im rho) = sum_j (cos, sin)(2 pi n . s_j) by direct NumPy sums."""
    theta = 2.0 * math.pi * (np.asarray(n, dtype=np.float64) @ s.T)
    return np.cos(theta).sum(1), np.sin(theta).sum(1)


def md_observe(r: np.ndarray, basis: np.ndarray, waves_n: np.ndarray, kvec: np.ndarray, nc: int,
               rho_prev: np.ndarray, wind: bool, corrected: bool) -> tuple:
    """(rho (w, 2), active (w,)) of one step: every constrained wave and, when
    ``wind``, the others from direct sums at s = r B^-1; exp(-i k . R_cm) when
    ``corrected``; inactive rows keep rho_prev."""
    w = waves_n.shape[0]
    s = r @ np.linalg.inv(basis)
    rcm = r.mean(axis=0)
    rows = np.arange(w) if wind else np.arange(nc)
    re, im = density_direct(s, waves_n[rows])
    rho = rho_prev.copy()
    new = np.stack([re, im], axis=-1)
    if corrected:
        ph = kvec[rows] @ rcm
        c, sn = np.cos(ph), np.sin(ph)
        new = np.stack([new[:, 0] * c + new[:, 1] * sn, new[:, 1] * c - new[:, 0] * sn], axis=-1)
    active = np.zeros(w, dtype=bool)
    active[rows] = True
    rho[rows] = new
    return rho, active


def md_winding(rho_prev, rho_new, wind_abs, wind_net, n_valid, active, n, floor):
    """One winding update: phase change atan2 of rho_new conj(rho_old), counted
    for active waves with |rho|^2 / n above ``floor`` at both ends."""
    o, q = rho_prev, rho_new
    delta = np.arctan2(q[:, 1] * o[:, 0] - q[:, 0] * o[:, 1], q[:, 0] * o[:, 0] + q[:, 1] * o[:, 1])
    s_old = (o ** 2).sum(1) / n
    s_new = (q ** 2).sum(1) / n
    ok = active & (s_old > floor) & (s_new > floor)
    keep = np.where(active[:, None], q, o)
    return keep, wind_abs + np.where(ok, np.abs(delta), 0.0), wind_net + np.where(ok, delta, 0.0), \
        n_valid + ok.astype(np.int64)
