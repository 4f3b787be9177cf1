"""MD checkpoints in the reference's file layout (``src/xla_cco/dynamics/checkpoint.py:47-205``).

An .npz (no pickles) holding every array of an ``MDState`` as ``leaf_000``,
``leaf_001``, ... in the state's flattening order (its fields in declaration
order, the ``snap`` and ``trace`` buffers' fields in place), the leaf count
``__n_leaves__`` (int64) and ``__meta__`` (0-d unicode, JSON). Files written
by the reference load here and the other way round. The PRNG key is stored as
uint32[2] per lane. Writes are atomic: ``<path>.tmp``, fsync, rename; an
unreadable or mismatched file raises ``CheckpointError`` (a ValueError).
"""

from __future__ import annotations

import contextlib
import dataclasses
import json
import os
import zipfile
from pathlib import Path
from typing import Any, Dict, List, Tuple

import numpy as np

from xla_cco.dynamics.state import MDState, RhoTrace, Snapshots

META_KEY = "__meta__"
COUNT_KEY = "__n_leaves__"
LEAF_FORMAT = "leaf_{:03d}"
TMP_SUFFIX = ".tmp"

_NESTED = {"snap": Snapshots, "trace": RhoTrace}


class CheckpointError(ValueError):
    """A checkpoint that is unreadable or does not match its template."""


def tmp_path_of(path: Path) -> Path:
    """The temporary file ``save_state`` renames over ``path``."""
    return Path(str(path) + TMP_SUFFIX)


def _host(x: Any) -> np.ndarray:
    return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)


def _leaf_paths() -> List[Tuple[str, ...]]:
    """Field paths of an MDState in flattening order."""
    out: List[Tuple[str, ...]] = []
    for f in dataclasses.fields(MDState):
        nested = _NESTED.get(f.name)
        if nested is None:
            out.append((f.name,))
        else:
            out.extend((f.name, g.name) for g in dataclasses.fields(nested))
    return out


def _leaves(state: MDState) -> List[np.ndarray]:
    leaves = []
    for path in _leaf_paths():
        obj = state
        for name in path:
            obj = getattr(obj, name)
        a = _host(obj)
        if path == ("key",) and a.dtype == np.int32:   # device keys travel as int32 bits
            a = a.view(np.uint32)
        leaves.append(a)
    return leaves


def _build(leaves: List[np.ndarray]) -> MDState:
    fields: Dict[str, Any] = {}
    nested: Dict[str, Dict[str, Any]] = {k: {} for k in _NESTED}
    for path, a in zip(_leaf_paths(), leaves):
        if len(path) == 1:
            fields[path[0]] = a
        else:
            nested[path[0]][path[1]] = a
    for name, cls in _NESTED.items():
        fields[name] = cls(**nested[name])
    return MDState(**fields)


def save_state(path: Path, state: MDState, meta: Dict[str, Any]) -> None:
    """Write ``state`` and ``meta`` to ``path`` atomically; on any error the
    temporary file is removed and ``path`` keeps its previous content.
    ``TypeError`` unless ``state`` is an MDState and ``meta`` a JSON dict."""
    if not isinstance(state, MDState):
        raise TypeError(f"state must be an MDState, got {type(state).__name__}")
    if not isinstance(meta, dict):
        raise TypeError(f"meta must be a dict, got {type(meta).__name__}")
    text = json.dumps(meta, sort_keys=True)
    arrays = {LEAF_FORMAT.format(i): a for i, a in enumerate(_leaves(state))}
    arrays[META_KEY] = np.asarray(text)
    arrays[COUNT_KEY] = np.int64(len(arrays) - 1)
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


def _meta_of(z: Any, path: Path) -> Dict[str, Any]:
    if META_KEY not in z.files or COUNT_KEY not in z.files:
        raise CheckpointError(f"{path} is not an MD checkpoint (no {META_KEY})")
    meta = json.loads(str(z[META_KEY][()]))
    if not isinstance(meta, dict):
        raise CheckpointError(f"{path}: metadata is not a JSON object")
    return meta


def _unreadable(path: Path, exc: Exception) -> CheckpointError:
    return CheckpointError(f"{path} is not a readable MD checkpoint (truncated or corrupt: "
                           f"{type(exc).__name__}: {exc})")  # fmt: skip


def read_meta(path: Path) -> Dict[str, Any]:
    """The metadata of a checkpoint (no template needed)."""
    try:
        with np.load(Path(path), allow_pickle=False) as z:
            return _meta_of(z, Path(path))
    except CheckpointError:
        raise
    except (zipfile.BadZipFile, EOFError, KeyError, ValueError) as exc:
        raise _unreadable(Path(path), exc) from exc


def load_state(path: Path, like: MDState) -> Tuple[MDState, Dict[str, Any]]:
    """(state, meta) of a checkpoint; the leaf count and every leaf's shape and
    dtype must match the template ``like`` (``CheckpointError`` otherwise)."""
    if not isinstance(like, MDState):
        raise TypeError(f"like must be an MDState, got {type(like).__name__}")
    want = _leaves(like)
    path = Path(path)
    try:
        with np.load(path, allow_pickle=False) as z:
            meta = _meta_of(z, path)
            count = int(z[COUNT_KEY])
            if count != len(want):
                raise CheckpointError(f"{path} holds {count} leaves; the template has {len(want)}")
            got = []
            for i, ref in enumerate(want):
                a = np.asarray(z[LEAF_FORMAT.format(i)])
                if a.shape != ref.shape or a.dtype != ref.dtype:
                    raise CheckpointError(f"{path} leaf {i}: stored {a.shape} {a.dtype}, "
                                          f"template {ref.shape} {ref.dtype}")  # fmt: skip
                got.append(a)
    except CheckpointError:
        raise
    except (zipfile.BadZipFile, EOFError, KeyError, ValueError) as exc:
        raise _unreadable(path, exc) from exc
    return _build(got), meta
