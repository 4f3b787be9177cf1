"""MD checkpoints (``src/xla_cco/dynamics/checkpoint.py:61-205``): an .npz of
every array of an ``MDState`` by field name plus a JSON metadata entry,
written atomically (temporary file, fsync, rename)."""

from __future__ import annotations

import contextlib
import dataclasses
import json
import os
import zipfile
from pathlib import Path
from typing import Any, Dict, Tuple

import numpy as np

from xla_cco.dynamics.state import MDState, RhoTrace, Snapshots

META_KEY = "__meta__"
TMP_SUFFIX = ".tmp"


class CheckpointError(ValueError):
    """A checkpoint that is unreadable or does not match its template."""


def tmp_path_of(path: Path) -> Path:
    return Path(str(path) + TMP_SUFFIX)


def _host(x: Any) -> np.ndarray:
    return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)


def _flat(state: MDState) -> Dict[str, np.ndarray]:
    out: Dict[str, np.ndarray] = {}
    for f in dataclasses.fields(state):
        v = getattr(state, f.name)
        if isinstance(v, (Snapshots, RhoTrace)):
            for g in dataclasses.fields(v):
                out[f"{f.name}.{g.name}"] = _host(getattr(v, g.name))
        else:
            out[f.name] = _host(v)
    if out["key"].dtype == np.int32:   # device keys travel as int32 bits
        out["key"] = out["key"].view(np.uint32)
    return out


def save_state(path: Path, state: MDState, meta: Dict[str, Any]) -> None:
    """Write ``state`` and ``meta`` to ``path``; on error ``path`` is untouched."""
    if not isinstance(state, MDState):
        raise TypeError(f"state must be an MDState, got {type(state).__name__}")
    if not isinstance(meta, dict):
        raise TypeError(f"meta must be a dict, got {type(meta).__name__}")
    arrays = _flat(state)
    arrays[META_KEY] = np.asarray(json.dumps(meta, sort_keys=True))
    path = Path(path)
    tmp = tmp_path_of(path)
    try:
        with open(tmp, "wb") as fh:
            np.savez(fh, **arrays)
            fh.flush()
            os.fsync(fh.fileno())
        os.replace(tmp, path)
    except BaseException:
        with contextlib.suppress(OSError):
            tmp.unlink()
        raise


def _open(path: Path):
    try:
        return np.load(Path(path), allow_pickle=False)
    except (OSError, ValueError, zipfile.BadZipFile, EOFError) as exc:
        raise CheckpointError(f"unreadable checkpoint {path}: {exc}") from exc


def read_meta(path: Path) -> Dict[str, Any]:
    """The metadata dict of a checkpoint."""
    with _open(path) as z:
        if META_KEY not in z.files:
            raise CheckpointError(f"{path}: no metadata")
        return json.loads(str(z[META_KEY]))


def load_state(path: Path, like: MDState) -> Tuple[MDState, Dict[str, Any]]:
    """(state, meta) of a checkpoint; every array must match ``like`` in
    shape and dtype (``CheckpointError`` otherwise)."""
    want = _flat(like)
    with _open(path) as z:
        try:
            got = {k: z[k] for k in want}
            meta = json.loads(str(z[META_KEY]))
        except (KeyError, ValueError, zipfile.BadZipFile) as exc:
            raise CheckpointError(f"{path}: {exc}") from exc
    for k, v in want.items():
        if got[k].shape != v.shape or got[k].dtype != v.dtype:
            raise CheckpointError(f"{path}: {k} is {got[k].dtype}{got[k].shape}, "
                                  f"expected {v.dtype}{v.shape}")  # fmt: skip
    snap = Snapshots(**{g.name: got[f"snap.{g.name}"] for g in dataclasses.fields(Snapshots)})
    trace = RhoTrace(**{g.name: got[f"trace.{g.name}"] for g in dataclasses.fields(RhoTrace)})
    plain = {f.name: got[f.name] for f in dataclasses.fields(MDState) if f.name not in ("snap", "trace")}
    return MDState(**plain, snap=snap, trace=trace), meta
