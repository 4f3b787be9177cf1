"""Ground-state driver: ``python -m xla_cco.cli.relax`` (the C++ ground/input mode).

What a user of the reference sees is kept: the options, validation
messages, output files, table layouts and log keys of
``src/xla_cco/cli/relax.py:101-164,488-546``. Behind them the driver is one
pipeline whose data stay on the GPU between reading and writing::

    ConfigPack --read--> host records, wrapped positions --one upload-->
    device positions --relax, --batch-size lanes per device call, results
    written into device buffers--> device results --success mask, Success
    gather, S(k), pair counts, nearest neighbours and their histogram, on the
    device--> one download (positions, energies, statuses, counts) --> files

Files written for prefix SAVE: ``SAVE.ConfigPack`` (relaxed),
``SAVE_InitConfig.ConfigPack`` (the wrapped input), ``SAVE_Success.ConfigPack``
(energy < ``--tol``), each with the C++ headers (cell size N^(1/d), basis =
unit basis x N^(1/d)); ``SAVE_Sk.txt``, ``SAVE_g2.txt`` and ``SAVE_Hp.txt``
of the Success set in the C++ four-column layout; ``SAVE_energies.npy``,
``SAVE_log.json`` and, when recording, ``SAVE_traj.npz``.

g2 and Hp use fixed uniform grids where C++ builds adaptive bins (g2 on
[0, 0.2 L] with ``--g2-bins``; Hp on [0, largest nearest-neighbour distance]
with ``--hp-bins``, every bin kept); S(k) uses the C++ binning (directions
|k| < 5, multiples to |k| <= 400). Success is energy < ``--tol`` only: an
L-BFGS lane ending with STATUS_LINESEARCH_FAIL far below the tolerance has
reached roundoff, which is the normal end. ``--device cpu`` is refused with a
RuntimeError: this build has no CPU path.
"""

from __future__ import annotations

import argparse
import collections
import dataclasses
import json
import sys
import time
from pathlib import Path
from typing import Any, Dict, Iterator, List, Sequence, Tuple, Union

import numpy as np

from xla_cco import _native
from xla_cco._device import require_gpu
from xla_cco.analysis.pairs import g2_from_histogram, nearest_neighbor_distances_batch, pair_distance_histogram
from xla_cco.analysis.structure import isotropic_structure_factor
from xla_cco.box import Box, cubic_box, wrap_fractional
from xla_cco.energy import make_stealthy_energy
from xla_cco.io.configpack import PackedConfig, read_configpack, stack_fractional, write_configpack
from xla_cco.io.tables import write_function_table
from xla_cco.kvectors import chi_from_count, enumerate_kvectors, k_outer_from_ka
from xla_cco.minimize import relax_device
from xla_cco.minimize import result as result_mod
from xla_cco.minimize.descent import DescentSettings
from xla_cco.minimize.lbfgs import LBFGSSettings

Settings = Union[DescentSettings, LBFGSSettings]

CPP_PARITY_TOL = 9.99999968e-21      # float32(1e-20) as a double: the C++ success threshold
UNIT_VOLUME_ATOL = 1e-12             # |det| tolerance of the two input cell conventions
G2_CUTOFF_FRACTION = 0.2             # g2 up to 0.2 L (C++ main.cpp)
SK_K_DIR_MAX, SK_K_MAX = 5.0, 400.0  # IsotropicStructureFactor(..., 5, 400)

_STATUS_NAME = {getattr(result_mod, k): k for k in dir(result_mod) if k.startswith("STATUS_")}

# ------------------------------------------------------------------ command line
_DESCRIPTION = (
    "Relax ConfigPack configurations to stealthy ground states (C++ ground/input mode) on "
    "the GPU. NOTE: C++ uses adaptive bins for g2 and Hp; here both are on fixed uniform "
    "grids (--g2-bins, --hp-bins), and Hp keeps all bins while C++ drops its last bin. "
    "Success is judged only by energy < --tol (see n_success in SAVE_log.json); status "
    "STATUS_LINESEARCH_FAIL with energy far below tol is the normal end of L-BFGS at "
    "roundoff, not a failure."
)

# (flag, argparse keywords): the reference driver's options, in its order
_OPTIONS: Tuple[Tuple[str, Dict[str, Any]], ...] = (
    ("--dim", dict(type=int, required=True, help="dimension d (1-3)")),
    ("--ka", dict(type=float, required=True, help="K2 * a (outer radius)")),
    ("--phi", dict(type=float, required=True, help="packing fraction")),
    ("--k1a", dict(type=float, default=0.0, help="K1 * a (default 0)")),
    ("--load", dict(type=Path, required=True, help="input pack prefix")),
    ("--input-basis", dict(choices=("auto", "unit", "scaled"), default="auto",
                           help="input cell convention: unit = unit-volume basis (C++ input "
                                "mode); scaled = basis already multiplied by N^(1/d), as this "
                                "driver writes its outputs; auto = accept either (default)")),
    ("--save", dict(type=Path, required=True, help="output prefix")),
    ("--method", dict(choices=("lbfgs", "descent"), default="lbfgs")),
    ("--tol", dict(type=float, default=1e-20,
                   help="success threshold on the energy, used verbatim as float64 "
                        f"(C++ parity value: {CPP_PARITY_TOL:.8e})")),
    ("--max-steps", dict(type=int, default=None,
                         help="evaluation budget: lbfgs max_evals_per_pass, descent max_evals")),
    ("--grow", dict(type=float, default=1.0, help="descent step growth")),
    ("--stop-tol", dict(type=float, default=0.0,
                        help="early-stopping energy (0 = C++ behaviour: never stop early)")),
    ("--batch-size", dict(type=int, default=1024, help="configs per call")),
    ("--chunk-size", dict(type=int, default=None,
                          help="k-chunk of the energy (accepted; the kernels do not chunk)")),
    ("--device", dict(choices=("gpu", "cpu"), default="gpu")),
    ("--record-every", dict(type=int, default=0, help="trajectory stride")),
    ("--max-records", dict(type=int, default=0, help="trajectory capacity")),
    ("--g2-bins", dict(type=int, default=200, help="fixed g2 grid bins")),
    ("--hp-bins", dict(type=int, default=200, help="fixed Hp grid bins")),
)  # fmt: skip


def build_parser() -> argparse.ArgumentParser:
    """The driver's argument parser (the reference driver's options)."""
    parser = argparse.ArgumentParser(prog="python -m xla_cco.cli.relax", description=_DESCRIPTION)
    for flag, spec in _OPTIONS:
        parser.add_argument(flag, **spec)
    return parser


def _argument_rules(a: argparse.Namespace) -> Iterator[Tuple[bool, str]]:
    """(condition that must hold, message if it does not), in checking order."""
    yield a.dim in (1, 2, 3), f"--dim must be 1, 2 or 3, got {a.dim}"
    yield a.ka > 0.0, f"--ka must be positive, got {a.ka}"
    yield a.phi > 0.0, f"--phi must be positive, got {a.phi}"
    yield 0.0 <= a.k1a < a.ka, f"need 0 <= --k1a < --ka, got {a.k1a}, {a.ka}"
    yield a.tol > 0.0, f"--tol must be positive, got {a.tol}"
    yield a.stop_tol >= 0.0, f"--stop-tol must be >= 0, got {a.stop_tol}"
    yield a.max_steps is None or a.max_steps >= 1, f"--max-steps must be >= 1, got {a.max_steps}"
    yield a.method != "lbfgs" or a.grow == 1.0, "--grow applies to --method descent only"
    yield a.grow >= 1.0, f"--grow must be >= 1, got {a.grow}"
    for name in ("batch_size", "g2_bins", "hp_bins"):
        yield getattr(a, name) >= 1, f"--{name.replace('_', '-')} must be >= 1"
    yield a.chunk_size is None or a.chunk_size >= 1, f"--chunk-size must be >= 1, got {a.chunk_size}"
    yield min(a.record_every, a.max_records) >= 0, "--record-every and --max-records must be >= 0"
    yield (a.record_every > 0) == (a.max_records > 0), \
        "--record-every and --max-records must both be positive"


def validate_args(args: argparse.Namespace) -> None:
    """``ValueError`` naming the option on the first inconsistent argument."""
    for holds, message in _argument_rules(args):
        if not holds:
            raise ValueError(message)


def select_device(device: str) -> str:
    """``"gpu"`` when a CUDA device is visible (``RuntimeError`` naming the
    cause otherwise); ``--device cpu`` is refused: there is no CPU path."""
    assert device in ("gpu", "cpu"), "device must be gpu or cpu"
    if device == "cpu":
        raise RuntimeError("requested --device cpu, but this build computes on the GPU only "
                           "(libcco.so, sm_100a); run with --device gpu")  # fmt: skip
    require_gpu()
    return "gpu"


# ------------------------------------------------------------------ input
def _unit_cell_divisor(index: int, basis: np.ndarray, n: int, convention: str) -> float:
    """What the stored basis is divided by to give the unit basis: 1 for a
    unit-volume cell (C++ input mode), N^(1/d) for a cell already scaled by it
    (this driver's own outputs); ``ValueError`` for any other volume or a
    convention the caller excluded."""
    det = abs(float(np.linalg.det(basis)))
    if abs(det - 1.0) <= UNIT_VOLUME_ATOL and convention in ("auto", "unit"):
        return 1.0
    if abs(det / n - 1.0) <= UNIT_VOLUME_ATOL * max(1.0, float(n)) and convention in ("auto", "scaled"):
        return float(n) ** (1.0 / basis.shape[0])
    raise ValueError(
        f"config {index}: input basis has |det| = {det!r}; with --input-basis {convention} the "
        "cell volume must be 1 (unit basis; C++ input mode multiplies it by N^(1/d)) or "
        f"N = {n} (basis already scaled by N^(1/d), as this driver writes outputs)")


def load_input(prefix: Path, dim: int, input_basis: str = "auto"
               ) -> Tuple[List[PackedConfig], np.ndarray, np.ndarray]:  # fmt: skip
    """(records with unit bases, (B, N, d) positions wrapped into [0, 1), unit basis).

    ``ValueError`` on an empty pack, a dimension other than ``dim``, mixed N or
    d, or a cell that fits neither accepted convention; ``FileNotFoundError``
    for a missing pack; ``TypeError`` on non-float64 positions.
    """
    assert input_basis in ("auto", "unit", "scaled"), "unknown input_basis"
    records = read_configpack(prefix)
    if not records:
        raise ValueError(f"no configurations in {prefix}")
    found = int(np.asarray(records[0].relative).shape[1])
    if found != dim:
        raise ValueError(f"--dim {dim} does not match pack dimension {found}")
    stacked, _ = stack_fractional(records)
    n = int(stacked.shape[1])
    unit = []
    for i, rec in enumerate(records):
        basis = np.asarray(rec.basis, dtype=np.float64)
        divisor = _unit_cell_divisor(i, basis, n, input_basis)
        unit.append(rec if divisor == 1.0 else dataclasses.replace(rec, basis=basis / divisor))
    return unit, wrap_fractional(stacked), np.asarray(unit[0].basis, dtype=np.float64)


# ------------------------------------------------------------------ physics and settings
def build_physics(unit_basis: np.ndarray, n: int, args: argparse.Namespace
                  ) -> Tuple[Box, Any, Dict[str, Any]]:  # fmt: skip
    """(box of side N^(1/d) over the unit basis, energy, info) with K1 = k1a / a
    and K2 = ka / a sharing one a (``ValueError`` below 2 particles or on an
    empty k-set)."""
    d = args.dim
    if n < 2:
        raise ValueError(f"need at least 2 particles, got N = {n}")
    side = float(n) ** (1.0 / d)
    cubic = np.array_equal(unit_basis, np.eye(d))
    box = cubic_box(n, d) if cubic else Box(basis=unit_basis * side)
    k_out = k_outer_from_ka(args.ka, args.phi, d)
    k_in = k_outer_from_ka(args.k1a, args.phi, d) if args.k1a > 0.0 else 0.0
    kset = enumerate_kvectors(np.asarray(box.basis), k_in, k_out)
    m = int(kset.n.shape[0])
    if m == 0:
        raise ValueError(f"empty k-set for K1={k_in}, K2={k_out}")
    info = dict(N=n, d=d, M=m, chi=chi_from_count(m, n, d), a=args.ka / k_out, K1=k_in, K2=k_out)
    return box, make_stealthy_energy(box, kset, chunk_size=args.chunk_size), info


# --method -> (settings class, field that --max-steps sets)
_MINIMIZERS = {"lbfgs": (LBFGSSettings, "max_evals_per_pass"), "descent": (DescentSettings, "max_evals")}


def make_settings(args: argparse.Namespace) -> Settings:
    """The minimizer settings the arguments select (reference defaults otherwise)."""
    cls, budget_field = _MINIMIZERS[args.method]
    fields: Dict[str, Any] = dict(energy_tol=args.stop_tol, record_every=args.record_every,
                                  max_records=args.max_records)  # fmt: skip
    if args.max_steps is not None:
        fields[budget_field] = args.max_steps
    if cls is DescentSettings:
        fields["grow"] = args.grow
    return cls(**fields)


# ------------------------------------------------------------------ device stages
_RESULT_FIELDS = ("s", "energy", "n_evals", "n_iters", "status")
_TRAJ_FIELDS = ("s", "energy", "step", "iteration", "count")


def _relax_on_device(energy: Any, s0: np.ndarray, settings: Settings, batch_size: int):
    """Upload every configuration once, relax ``batch_size`` lanes per device
    call, and keep every result on the device: a dict of CUDA tensors with the
    whole batch on the leading axis (trajectory fields prefixed ``traj_``)."""
    import torch

    b = s0.shape[0]
    s_dev = torch.from_numpy(np.ascontiguousarray(s0)).pin_memory().cuda(non_blocking=True)
    results: Dict[str, Any] = {}
    for lo in range(0, b, batch_size):
        hi = min(b, lo + batch_size)
        part = relax_device(energy, s_dev[lo:hi], settings)
        keys = [(k, k) for k in _RESULT_FIELDS] + [(f"traj_{k}", f"traj_{k}") for k in _TRAJ_FIELDS]
        for dst, src in keys:
            if src not in part:
                continue
            if dst not in results:
                results[dst] = torch.empty((b,) + tuple(part[src].shape[1:]), dtype=part[src].dtype,
                                           device=s_dev.device)  # fmt: skip
            results[dst][lo:hi] = part[src]
    return s_dev, results


def _histogram_on_device(values: Any, edges: np.ndarray) -> np.ndarray:
    """np.histogram counts of a CUDA tensor over ``edges``: bins [e_k, e_k+1),
    the last one closed, values outside [e_0, e_-1] dropped - by comparing
    against the same edge values (torch.bucketize), so the counts equal
    np.histogram's."""
    import torch

    e = torch.from_numpy(np.asarray(edges, dtype=np.float64)).to(values.device)
    x = values.reshape(-1)
    idx = torch.bucketize(x, e, right=True) - 1          # e[idx] <= x < e[idx + 1]
    idx = torch.where(x == e[-1], torch.full_like(idx, e.numel() - 2), idx)
    keep = (idx >= 0) & (idx < e.numel() - 1)
    return torch.bincount(idx[keep], minlength=e.numel() - 1).cpu().numpy()


def table_columns(edges: np.ndarray, values: np.ndarray, counts: np.ndarray) -> List[np.ndarray]:
    """The C++ g2 / Hp table columns: bin centre, value, half-width,
    value / sqrt(count) (0 for an empty bin)."""
    counts = np.asarray(counts, dtype=np.float64)
    err = np.divide(values, np.sqrt(counts), out=np.zeros_like(values), where=counts > 0)
    return [0.5 * (edges[1:] + edges[:-1]), values, 0.5 * np.diff(edges), err]


def _analyses_on_device(s_ok: Any, box: Box, args: argparse.Namespace) -> Dict[str, List[np.ndarray]]:
    """S(k), g2 and Hp tables of the Success set, computed from its device copy."""
    b, n, d = (int(x) for x in s_ok.shape)
    side = float(n) ** (1.0 / d)
    tables = {"Sk": list(isotropic_structure_factor(s_ok, box, SK_K_DIR_MAX, SK_K_MAX))}
    g2_edges = np.linspace(0.0, G2_CUTOFF_FRACTION * side, args.g2_bins + 1)
    pairs = pair_distance_histogram(s_ok, box, g2_edges)
    g2 = g2_from_histogram(pairs, g2_edges, n, b, float(n), d)
    tables["g2"] = table_columns(g2_edges, g2, pairs)
    nn = nearest_neighbor_distances_batch(s_ok, box)
    hp_edges = np.linspace(0.0, max(float(nn.max().item()), 1e-12), args.hp_bins + 1)
    hp_counts = _histogram_on_device(nn, hp_edges)
    tables["Hp"] = table_columns(hp_edges, hp_density(hp_counts, hp_edges), hp_counts)
    return tables


def hp_density(counts: np.ndarray, edges: np.ndarray) -> np.ndarray:
    """Nearest-neighbour probability density per bin: count / total / width."""
    counts = np.asarray(counts, dtype=np.float64)
    assert counts.shape == (edges.size - 1,), "counts must match the bins"
    total = counts.sum()
    assert total > 0.0, "need at least one nearest-neighbour distance"
    return counts / total / np.diff(edges)


# ------------------------------------------------------------------ output
def pack_configs(template: Sequence[PackedConfig], s: np.ndarray, side: float) -> List[PackedConfig]:
    """Output records with the C++ headers: cell size N^(1/d), basis = unit basis x N^(1/d)."""
    assert len(template) == s.shape[0], "one template per configuration"
    out = []
    for rec, rel in zip(template, s):
        basis = np.asarray(rec.basis, dtype=np.float64) * side
        out.append(PackedConfig(basis, np.ascontiguousarray(rel, dtype=np.float64), side, rec.names))
    return out


def success_mask(energy: np.ndarray, tol: float) -> np.ndarray:
    """Strictly energy < tol (the C++ ``E < E_max``)."""
    assert tol > 0.0, "tol must be positive"
    return np.asarray(energy) < tol


def summarize(out: Dict[str, np.ndarray], tol: float) -> Dict[str, Any]:
    """Log entries: counts per status name, the success count, n_evals statistics."""
    tally = collections.Counter(int(c) for c in np.asarray(out["status"]).ravel())
    evals = np.asarray(out["n_evals"])
    return {
        "status_counts": {_STATUS_NAME.get(c, f"STATUS_{c}"): k for c, k in sorted(tally.items())},
        "n_success": int(success_mask(out["energy"], tol).sum()),
        "n_evals": {"min": int(evals.min()), "mean": float(evals.mean()),
                    "median": float(np.median(evals)), "max": int(evals.max())},
    }  # fmt: skip


def _jsonable(value: Any) -> Any:
    if isinstance(value, Path):
        return str(value)
    raise TypeError(f"not JSON serializable: {type(value).__name__}")


# ------------------------------------------------------------------ driver
def run(args: argparse.Namespace) -> Dict[str, Any]:
    """Run the driver: read, relax and analyse on the device, write every
    output; returns the log (also written to SAVE_log.json)."""
    clock = [time.perf_counter()]
    validate_args(args)
    platform = select_device(args.device)
    records, s0, unit_basis = load_input(args.load, args.dim, args.input_basis)
    n = int(s0.shape[1])
    box, energy, info = build_physics(unit_basis, n, args)
    settings = make_settings(args)
    clock.append(time.perf_counter())
    print(f"relaxing {s0.shape[0]} configs: N={n} M={info['M']} on {platform}", flush=True)

    s_dev, dev = _relax_on_device(energy, s0, settings, args.batch_size)
    ok_dev = dev["energy"] < args.tol
    tables = None
    if bool(ok_dev.any()):
        tables = _analyses_on_device(dev["s"][ok_dev], box, args)
    host = {k: v.cpu().numpy() for k, v in dev.items()}   # the one download
    del s_dev
    clock.append(time.perf_counter())

    save = str(args.save)
    Path(save).parent.mkdir(parents=True, exist_ok=True)
    side = float(n) ** (1.0 / args.dim)
    ok = success_mask(host["energy"], args.tol)
    write_configpack(Path(save), pack_configs(records, host["s"], side))
    write_configpack(Path(save + "_InitConfig"), pack_configs(records, s0, side))
    np.save(save + "_energies.npy", host["energy"])
    log = summarize(host, args.tol)
    if tables is None:
        log["analysis"] = "skipped: no Success configurations"
    else:
        kept = [rec for rec, flag in zip(records, ok) if flag]
        write_configpack(Path(save + "_Success"), pack_configs(kept, host["s"][ok], side))
        for name, columns in tables.items():
            write_function_table(Path(f"{save}_{name}.txt"), columns)
        log.update(analysis="written", sk_nan_error_bins=int(np.isnan(tables["Sk"][3]).sum()))
    traj = {k[len("traj_"):]: v for k, v in host.items() if k.startswith("traj_")}
    if traj:
        np.savez(save + "_traj.npz", **traj)
    clock.append(time.perf_counter())
    log.update(
        args=vars(args), **info, tol=args.tol, method=args.method,
        settings=dataclasses.asdict(settings), n_configs=int(s0.shape[0]),
        wall_seconds=dict(zip(("setup", "relax", "output"), np.diff(clock).tolist())),
        jax_version=None,   # key kept for readers of the reference's log; there is no JAX here
        engine=f"libcco ABI {_native.load().cco_abi_version()} (CUDA sm_100a)", device=platform,
    )  # fmt: skip
    Path(save + "_log.json").write_text(json.dumps(log, indent=2, default=_jsonable) + "\n")
    return log


def main(argv: Sequence[str] | None = None) -> int:
    parsed = build_parser().parse_args(argv)
    try:
        log = run(parsed)
    except (ValueError, TypeError, RuntimeError, OSError) as exc:
        print(f"ERROR: {exc}", file=sys.stderr, flush=True)
        return 1
    print(json.dumps(log, indent=2, default=_jsonable), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
