"""Ground-state driver: ``python -m xla_cco.cli.relax`` (the C++ ground/input mode).

Mirrors ``src/xla_cco/cli/relax.py:101-560`` of the reference: the same
options, validation messages, output files and log keys. It reads a
ConfigPack (``--load``), relaxes every configuration on the GPU with the
batched device minimizers, and writes for prefix SAVE:

* ``SAVE.ConfigPack`` (relaxed), ``SAVE_InitConfig.ConfigPack`` (the wrapped
  input) and ``SAVE_Success.ConfigPack`` (energy < ``--tol``), with the C++
  headers (cell size N^(1/d), basis = unit basis x N^(1/d));
* ``SAVE_Sk.txt``, ``SAVE_g2.txt``, ``SAVE_Hp.txt`` for the Success set in
  the C++ four-column layout;
* ``SAVE_energies.npy``, ``SAVE_log.json`` and, when recording,
  ``SAVE_traj.npz``.

Tables: g2 ``r_mid, g2, half-width, g2/sqrt(count)`` and Hp ``r_mid,
count/total/width, half-width, p/sqrt(count)`` (PairCorrelation.cpp). As in
the reference, g2 and Hp use FIXED uniform grids where C++ builds adaptive
bins (g2 on [0, 0.2 L] with ``--g2-bins``; Hp on [0, largest nearest-neighbour
distance] with ``--hp-bins``, all bins kept); S(k) uses the C++ binning
(``IsotropicStructureFactor`` with 5, 400).

Success is energy < ``--tol`` only. L-BFGS ending with STATUS_LINESEARCH_FAIL
far below tol is the normal end at roundoff, not a failure.

This build computes on the GPU only: ``--device cpu`` is refused with a
RuntimeError (there is no CPU path to fall back to).
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import sys
import time
from pathlib import Path
from typing import Any, Dict, List, Sequence, Tuple, Union

import numpy as np

from xla_cco import _native
from xla_cco._device import require_gpu
from xla_cco.analysis.pairs import (
    g2_from_histogram,
    nearest_neighbor_distances,
    pair_distance_histogram,
)
from xla_cco.analysis.structure import isotropic_structure_factor
from xla_cco.box import Box, cubic_box, wrap_fractional
from xla_cco.energy import make_stealthy_energy
from xla_cco.io.configpack import PackedConfig, read_configpack, stack_fractional, write_configpack
from xla_cco.io.tables import write_function_table
from xla_cco.kvectors import chi_from_count, enumerate_kvectors, k_outer_from_ka
from xla_cco.minimize import relax
from xla_cco.minimize import result as result_mod
from xla_cco.minimize.descent import DescentSettings
from xla_cco.minimize.lbfgs import LBFGSSettings

Settings = Union[DescentSettings, LBFGSSettings]

CPP_PARITY_TOL = 9.99999968e-21      # float32(1e-20) as a double: the C++ threshold
UNIT_VOLUME_ATOL = 1e-12
G2_CUTOFF_FRACTION = 0.2             # g2 up to 0.2 L (C++ main.cpp)
SK_K_DIR_MAX = 5.0                   # IsotropicStructureFactor(..., 5, 400)
SK_K_MAX = 400.0
STATUS_NAMES: Dict[int, str] = {
    getattr(result_mod, k): k for k in dir(result_mod) if k.startswith("STATUS_")
}


def build_parser() -> argparse.ArgumentParser:
    """The driver's argument parser (options of the reference driver)."""
    p = argparse.ArgumentParser(
        prog="python -m xla_cco.cli.relax",
        description=(
            "Relax ConfigPack configurations to stealthy ground states (C++ ground/input "
            "mode) on the GPU. NOTE: C++ uses adaptive bins for g2 and Hp; here both are on "
            "fixed uniform grids (--g2-bins, --hp-bins), and Hp keeps all bins while C++ "
            "drops its last bin. Success is judged only by energy < --tol (see n_success in "
            "SAVE_log.json); status STATUS_LINESEARCH_FAIL with energy far below tol is the "
            "normal end of L-BFGS at roundoff, not a failure."
        ),
    )  # fmt: skip
    p.add_argument("--dim", type=int, required=True, help="dimension d (1-3)")
    p.add_argument("--ka", type=float, required=True, help="K2 * a (outer radius)")
    p.add_argument("--phi", type=float, required=True, help="packing fraction")
    p.add_argument("--k1a", type=float, default=0.0, help="K1 * a (default 0)")
    p.add_argument("--load", type=Path, required=True, help="input pack prefix")
    p.add_argument("--input-basis", choices=("auto", "unit", "scaled"), default="auto",
                   help="input cell convention: unit = unit-volume basis (C++ input mode); "
                   "scaled = basis already multiplied by N^(1/d), as this driver writes its "
                   "outputs; auto = accept either (default)")  # fmt: skip
    p.add_argument("--save", type=Path, required=True, help="output prefix")
    p.add_argument("--method", choices=("lbfgs", "descent"), default="lbfgs")
    p.add_argument("--tol", type=float, default=1e-20,
                   help="success threshold on the energy, used verbatim as float64 "
                   f"(C++ parity value: {CPP_PARITY_TOL:.8e})")  # fmt: skip
    p.add_argument("--max-steps", type=int, default=None,
                   help="evaluation budget: lbfgs max_evals_per_pass, descent max_evals")
    p.add_argument("--grow", type=float, default=1.0, help="descent step growth")
    p.add_argument("--stop-tol", type=float, default=0.0,
                   help="early-stopping energy (0 = C++ behaviour: never stop early)")
    p.add_argument("--batch-size", type=int, default=1024, help="configs per call")
    p.add_argument("--chunk-size", type=int, default=None,
                   help="k-chunk of the energy (accepted; the kernels do not chunk)")
    p.add_argument("--device", choices=("gpu", "cpu"), default="gpu")
    p.add_argument("--record-every", type=int, default=0, help="trajectory stride")
    p.add_argument("--max-records", type=int, default=0, help="trajectory capacity")
    p.add_argument("--g2-bins", type=int, default=200, help="fixed g2 grid bins")
    p.add_argument("--hp-bins", type=int, default=200, help="fixed Hp grid bins")
    return p


def validate_args(args: argparse.Namespace) -> None:
    """``ValueError`` naming the option on inconsistent arguments."""
    if args.dim not in (1, 2, 3):
        raise ValueError(f"--dim must be 1, 2 or 3, got {args.dim}")
    if not args.ka > 0.0:
        raise ValueError(f"--ka must be positive, got {args.ka}")
    if not args.phi > 0.0:
        raise ValueError(f"--phi must be positive, got {args.phi}")
    if not 0.0 <= args.k1a < args.ka:
        raise ValueError(f"need 0 <= --k1a < --ka, got {args.k1a}, {args.ka}")
    if not args.tol > 0.0:
        raise ValueError(f"--tol must be positive, got {args.tol}")
    if args.stop_tol < 0.0:
        raise ValueError(f"--stop-tol must be >= 0, got {args.stop_tol}")
    if args.max_steps is not None and args.max_steps < 1:
        raise ValueError(f"--max-steps must be >= 1, got {args.max_steps}")
    if args.method == "lbfgs" and args.grow != 1.0:
        raise ValueError("--grow applies to --method descent only")
    if args.grow < 1.0:
        raise ValueError(f"--grow must be >= 1, got {args.grow}")
    for name in ("batch_size", "g2_bins", "hp_bins"):
        if getattr(args, name) < 1:
            raise ValueError(f"--{name.replace('_', '-')} must be >= 1")
    if args.chunk_size is not None and args.chunk_size < 1:
        raise ValueError(f"--chunk-size must be >= 1, got {args.chunk_size}")
    if min(args.record_every, args.max_records) < 0:
        raise ValueError("--record-every and --max-records must be >= 0")
    if (args.record_every > 0) != (args.max_records > 0):
        raise ValueError("--record-every and --max-records must both be positive")


def select_device(device: str) -> str:
    """Check the requested device and return its platform name ("gpu").

    ``--device gpu`` needs a CUDA device (``RuntimeError`` with the cause
    otherwise); ``--device cpu`` is refused: this build has no CPU path.
    """
    assert device in ("gpu", "cpu"), "device must be gpu or cpu"
    if device == "cpu":
        raise RuntimeError("requested --device cpu, but this build computes on the GPU only "
                           "(libcco.so, sm_100a); run with --device gpu")  # fmt: skip
    require_gpu()
    return "gpu"


def load_input(prefix: Path, dim: int, input_basis: str = "auto"
               ) -> Tuple[List[PackedConfig], np.ndarray, np.ndarray]:  # fmt: skip
    """(unit-basis configs, (B, N, d) wrapped fractional positions, unit basis).

    ``input_basis``: "unit" (|det| = 1, the C++ input mode), "scaled"
    (|det| = N: basis times N^(1/d), this driver's output convention) or
    "auto" (either); scaled bases are divided by N^(1/d). ``ValueError`` on a
    dimension mismatch, mixed N or d, or a cell volume that matches neither
    accepted convention; ``TypeError`` on non-float64 positions.
    """
    assert input_basis in ("auto", "unit", "scaled"), "unknown input_basis"
    configs = read_configpack(prefix)
    if not configs:
        raise ValueError(f"no configurations in {prefix}")
    d_pack = int(np.asarray(configs[0].relative).shape[1])
    if d_pack != dim:
        raise ValueError(f"--dim {dim} does not match pack dimension {d_pack}")
    s0, _ = stack_fractional(configs)
    s0 = wrap_fractional_batch(s0)
    n = int(s0.shape[1])
    side = float(n) ** (1.0 / dim)
    unit = []
    for i, c in enumerate(configs):
        det = abs(float(np.linalg.det(np.asarray(c.basis))))
        is_unit = abs(det - 1.0) <= UNIT_VOLUME_ATOL
        is_scaled = abs(det / n - 1.0) <= UNIT_VOLUME_ATOL * max(1.0, float(n))
        if is_unit and input_basis in ("auto", "unit"):
            unit.append(c)
        elif is_scaled and input_basis in ("auto", "scaled"):
            unit.append(dataclasses.replace(c, basis=np.asarray(c.basis, dtype=np.float64) / side))
        else:
            raise ValueError(
                f"config {i}: input basis has |det| = {det!r}; with --input-basis {input_basis} "
                "the cell volume must be 1 (unit basis; C++ input mode multiplies it by N^(1/d)) "
                f"or N = {n} (basis already scaled by N^(1/d), as this driver writes outputs)")
    return unit, s0, np.asarray(unit[0].basis, dtype=np.float64)


def build_physics(unit_basis: np.ndarray, n: int, args: argparse.Namespace
                  ) -> Tuple[Box, Any, Dict[str, Any]]:  # fmt: skip
    """(box, energy, info) with K1 = k1a / a and K2 = ka / a."""
    d = args.dim
    if n < 2:
        raise ValueError(f"need at least 2 particles, got N = {n}")
    side = float(n) ** (1.0 / d)
    box = cubic_box(n, d) if np.array_equal(unit_basis, np.eye(d)) else Box(basis=unit_basis * side)
    k2 = k_outer_from_ka(args.ka, args.phi, d)
    k1 = k_outer_from_ka(args.k1a, args.phi, d) if args.k1a > 0.0 else 0.0
    kset = enumerate_kvectors(np.asarray(box.basis), k1, k2)
    m = int(kset.n.shape[0])
    if m == 0:
        raise ValueError(f"empty k-set for K1={k1}, K2={k2}")
    energy = make_stealthy_energy(box, kset, chunk_size=args.chunk_size)
    info = {"N": n, "d": d, "M": m, "chi": chi_from_count(m, n, d), "a": args.ka / k2,
            "K1": k1, "K2": k2}  # fmt: skip
    return box, energy, info


def make_settings(args: argparse.Namespace) -> Settings:
    """Minimizer settings selected by the arguments."""
    common: Dict[str, Any] = {"energy_tol": args.stop_tol, "record_every": args.record_every,
                              "max_records": args.max_records}  # fmt: skip
    if args.method == "lbfgs":
        if args.max_steps is not None:
            common["max_evals_per_pass"] = args.max_steps
        return LBFGSSettings(**common)
    if args.max_steps is not None:
        common["max_evals"] = args.max_steps
    return DescentSettings(grow=args.grow, **common)


def relax_batches(energy: Any, s0: np.ndarray, settings: Settings, batch_size: int
                  ) -> Dict[str, np.ndarray]:  # fmt: skip
    """Relax ``batch_size`` configurations per device call; concatenated host arrays."""
    assert s0.ndim == 3 and batch_size >= 1, "bad shapes"
    parts: List[Dict[str, np.ndarray]] = []
    for lo in range(0, s0.shape[0], batch_size):
        res = relax(energy, np.ascontiguousarray(s0[lo:lo + batch_size]), settings)
        part = {"s": wrap_fractional_batch(np.asarray(res.s)), "energy": np.asarray(res.energy),
                "n_evals": np.asarray(res.n_evals), "n_iters": np.asarray(res.n_iters),
                "status": np.asarray(res.status)}  # fmt: skip
        if res.trajectory is not None:
            for name in ("s", "energy", "step", "iteration", "count"):
                part[f"traj_{name}"] = np.asarray(getattr(res.trajectory, name))
        parts.append(part)
    return {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}


def wrap_fractional_batch(s: np.ndarray) -> np.ndarray:
    """Wrap a (b, n, d) batch of fractional positions into [0, 1)."""
    assert np.ndim(s) == 3, "s must have shape (b, n, d)"
    return wrap_fractional(np.asarray(s))


def pack_configs(template: Sequence[PackedConfig], s: np.ndarray, side: float
                 ) -> List[PackedConfig]:  # fmt: skip
    """C++ output records: cell size N^(1/d), basis = unit basis x N^(1/d)."""
    assert len(template) == s.shape[0], "one template per configuration"
    return [PackedConfig(basis=np.asarray(c.basis, dtype=np.float64) * side,
                         relative=np.ascontiguousarray(rel, dtype=np.float64),
                         cell_size=side, names=c.names)
            for c, rel in zip(template, s)]  # fmt: skip


def hp_table(counts: np.ndarray, edges: np.ndarray) -> np.ndarray:
    """(bins, 4) Hp table: r_mid, count / total / width, half-width, p / sqrt(count)."""
    counts = np.asarray(counts, dtype=np.float64)
    assert counts.shape == (edges.size - 1,), "counts must match the bins"
    total = counts.sum()
    assert total > 0.0, "need at least one nearest-neighbour distance"
    half = 0.5 * np.diff(edges)
    p = counts / total / (2.0 * half)
    err = np.divide(p, np.sqrt(counts), out=np.zeros_like(p), where=counts > 0)
    return np.stack([0.5 * (edges[1:] + edges[:-1]), p, half, err], axis=1)


def g2_table(g2: np.ndarray, counts: np.ndarray, edges: np.ndarray) -> np.ndarray:
    """(bins, 4) g2 table: r_mid, g2, half-width, g2 / sqrt(count)."""
    counts = np.asarray(counts, dtype=np.float64)
    assert g2.shape == counts.shape == (edges.size - 1,), "shapes must match"
    err = np.divide(g2, np.sqrt(counts), out=np.zeros_like(g2), where=counts > 0)
    return np.stack([0.5 * (edges[1:] + edges[:-1]), g2, 0.5 * np.diff(edges), err], axis=1)


def _write_table(path: Path, table: np.ndarray) -> None:
    write_function_table(path, [table[:, j] for j in range(table.shape[1])])


def write_analyses(prefix: str, s_succ: np.ndarray, box: Box, args: argparse.Namespace
                   ) -> Dict[str, Any]:  # fmt: skip
    """Write S(k), g2 and Hp of the Success set; return the log entries."""
    n, d = s_succ.shape[1], s_succ.shape[2]
    side = float(n) ** (1.0 / d)
    k_mod, s_k, k_err, s_err = isotropic_structure_factor(s_succ, box, SK_K_DIR_MAX, SK_K_MAX)
    n_nan = int(np.isnan(s_err).sum())
    write_function_table(Path(prefix + "_Sk.txt"), [k_mod, s_k, k_err, s_err])

    g2_edges = np.linspace(0.0, G2_CUTOFF_FRACTION * side, args.g2_bins + 1)
    g2_counts = np.zeros(args.g2_bins, dtype=np.int64)
    nn: List[np.ndarray] = []
    for lo in range(0, s_succ.shape[0], args.batch_size):
        chunk = np.ascontiguousarray(s_succ[lo:lo + args.batch_size])
        g2_counts += pair_distance_histogram(chunk, box, g2_edges)
        nn += [np.asarray(nearest_neighbor_distances(c, box)) for c in chunk]
    g2 = g2_from_histogram(g2_counts, g2_edges, n, s_succ.shape[0], float(n), d)
    _write_table(Path(prefix + "_g2.txt"), g2_table(g2, g2_counts, g2_edges))

    nn_all = np.concatenate(nn)
    hp_edges = np.linspace(0.0, float(max(nn_all.max(), 1e-12)), args.hp_bins + 1)
    hp_counts, _ = np.histogram(nn_all, bins=hp_edges)
    _write_table(Path(prefix + "_Hp.txt"), hp_table(hp_counts, hp_edges))
    return {"analysis": "written", "sk_nan_error_bins": n_nan}


def success_mask(energy: np.ndarray, tol: float) -> np.ndarray:
    """Strictly energy < tol (the C++ ``E < E_max``)."""
    assert tol > 0.0, "tol must be positive"
    return np.asarray(energy) < tol


def summarize(out: Dict[str, np.ndarray], tol: float) -> Dict[str, Any]:
    """Status counts, success count and n_evals statistics."""
    status = out["status"]
    counts = {STATUS_NAMES.get(int(c), f"STATUS_{int(c)}"): int((status == c).sum())
              for c in np.unique(status)}  # fmt: skip
    ev = out["n_evals"]
    return {"status_counts": counts, "n_success": int(success_mask(out["energy"], tol).sum()),
            "n_evals": {"min": int(ev.min()), "mean": float(ev.mean()),
                        "median": float(np.median(ev)), "max": int(ev.max())}}  # fmt: skip


def _jsonable(value: Any) -> Any:
    if isinstance(value, Path):
        return str(value)
    raise TypeError(f"not JSON serializable: {type(value).__name__}")


def run(args: argparse.Namespace) -> Dict[str, Any]:
    """Run the driver, write every output and return the summary (the log)."""
    validate_args(args)
    t0 = time.perf_counter()
    platform = select_device(args.device)
    configs, s0, unit_basis = load_input(args.load, args.dim, args.input_basis)
    n = int(s0.shape[1])
    box, energy, info = build_physics(unit_basis, n, args)
    settings = make_settings(args)
    t_setup = time.perf_counter()
    print(f"relaxing {s0.shape[0]} configs: N={n} M={info['M']} on {platform}", flush=True)
    out = relax_batches(energy, s0, settings, args.batch_size)
    t_relax = time.perf_counter()

    prefix = str(args.save)
    Path(prefix).parent.mkdir(parents=True, exist_ok=True)
    side = float(n) ** (1.0 / args.dim)
    ok = success_mask(out["energy"], args.tol)
    write_configpack(Path(prefix), pack_configs(configs, out["s"], side))
    write_configpack(Path(prefix + "_InitConfig"), pack_configs(configs, s0, side))
    np.save(prefix + "_energies.npy", out["energy"])
    summary = summarize(out, args.tol)
    if ok.any():
        succ = [c for c, f in zip(configs, ok) if f]
        write_configpack(Path(prefix + "_Success"), pack_configs(succ, out["s"][ok], side))
        summary.update(write_analyses(prefix, out["s"][ok], box, args))
    else:
        summary["analysis"] = "skipped: no Success configurations"
    if "traj_s" in out:
        np.savez(prefix + "_traj.npz", **{k[5:]: v for k, v in out.items() if k.startswith("traj_")})
    t_end = time.perf_counter()
    summary.update({
        "args": vars(args), **info, "tol": args.tol, "method": args.method,
        "settings": dataclasses.asdict(settings), "n_configs": int(s0.shape[0]),
        "wall_seconds": {"setup": t_setup - t0, "relax": t_relax - t_setup,
                         "output": t_end - t_relax},
        "jax_version": None,   # key kept for readers of the reference log; no JAX here
        "engine": f"libcco ABI {_native.load().cco_abi_version()} (CUDA sm_100a)",
        "device": platform,
    })  # fmt: skip
    Path(prefix + "_log.json").write_text(json.dumps(summary, indent=2, default=_jsonable) + "\n")
    return summary


def main(argv: Sequence[str] | None = None) -> int:
    parsed = build_parser().parse_args(argv)
    try:
        result = run(parsed)
    except (ValueError, TypeError, RuntimeError, OSError) as exc:
        print(f"ERROR: {exc}", file=sys.stderr, flush=True)
        return 1
    print(json.dumps(result, indent=2, default=_jsonable), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
