"""ConfigPack reader and writer (the C++ binary configuration format).

Mirrors ``src/xla_cco/io/configpack.py:60-263`` of the reference: same
names, arguments, file layout and exceptions.

A pack is two files for a prefix P:

* ``P.ConfigPack``: the records back to back. One record is, little-endian,
  ``u16 d``, ``f64 cell_size``, ``f64 basis[d][d]`` (rows = lattice
  vectors), ``i32 N``, then N times (``f64 x[d]`` fractional position,
  4-byte name);
* ``P.ConfigPackIndex``: ``i64 count`` followed by ``count`` i64 byte
  offsets of the records.

The layout is fixed by the C++ program that shares these files, so it is the
reference's byte for byte. Positions are fractional; the C++ box is the basis
times N^(1/d).
"""

from __future__ import annotations

import dataclasses
import os
import struct
from pathlib import Path
from typing import List, Optional, Sequence, Tuple

import numpy as np

PACK_SUFFIX = ".ConfigPack"
INDEX_SUFFIX = ".ConfigPackIndex"
MAX_DIMENSION = 4     # the C++ MaxDimension
NAME_BYTES = 4
_UNIT_RTOL = 1e-12    # agreement of unit-volume bases across a stack


@dataclasses.dataclass(frozen=True)
class PackedConfig:
    """One stored configuration: (d, d) basis, (N, d) fractional positions,
    the cell size field and one 4-byte name per particle."""

    basis: np.ndarray
    relative: np.ndarray
    cell_size: float
    names: Tuple[bytes, ...]


def _files(prefix: Path) -> Tuple[Path, Path]:
    return Path(f"{prefix}{PACK_SUFFIX}"), Path(f"{prefix}{INDEX_SUFFIX}")


def _record_dtype(d: int) -> np.dtype:
    return np.dtype([("x", "<f8", (d,)), ("name", "V4")])


def _offsets(index_path: Path) -> np.ndarray:
    raw = np.fromfile(index_path, dtype="<i8")
    if raw.size == 0:
        raise ValueError(f"truncated index (no count): {index_path}")
    count = int(raw[0])
    if count < 0 or raw.size - 1 != count:
        raise ValueError(f"index {index_path} declares {count} configs but holds "
                         f"{raw.size - 1} offsets")  # fmt: skip
    return raw[1:]


def _decode(buf: memoryview, at: int) -> PackedConfig:
    size = len(buf)
    if at < 0 or at + 2 > size:
        raise ValueError(f"offset {at} outside pack ({size} B)")
    (d,) = struct.unpack_from("<H", buf, at)
    if not 1 <= d <= MAX_DIMENSION:
        raise ValueError(f"bad dimension {d} at offset {at}")
    head = 8 + 8 * d * d + 4
    pos = at + 2
    if pos + head > size:
        raise ValueError(f"truncated header at offset {at}")
    (cell,) = struct.unpack_from("<d", buf, pos)
    basis = np.frombuffer(buf, dtype="<f8", count=d * d, offset=pos + 8).reshape(d, d)
    (n,) = struct.unpack_from("<i", buf, pos + 8 + 8 * d * d)
    if n < 0:
        raise ValueError(f"negative particle count {n} at offset {at}")
    pos += head
    rec = _record_dtype(d)
    end = pos + n * rec.itemsize
    if end > size:
        raise ValueError(f"config at offset {at} overruns pack ({end} > {size} B)")
    recs = np.frombuffer(buf, dtype=rec, count=n, offset=pos)
    return PackedConfig(
        basis=np.array(basis, dtype=np.float64),
        relative=np.array(recs["x"], dtype=np.float64).reshape(n, d),
        cell_size=float(cell),
        names=tuple(bytes(v) for v in recs["name"]),
    )  # fmt: skip


def _encode(cfg: PackedConfig) -> bytes:
    basis, rel = np.asarray(cfg.basis), np.asarray(cfg.relative)
    for label, arr in (("basis", basis), ("relative", rel)):
        if arr.dtype != np.float64:
            raise TypeError(f"{label} must be float64, got {arr.dtype}")
    if rel.ndim != 2 or not 1 <= rel.shape[1] <= MAX_DIMENSION:
        raise ValueError(f"relative must be (N, d) with d in 1..{MAX_DIMENSION}; got {rel.shape}")
    n, d = rel.shape
    if basis.shape != (d, d):
        raise ValueError(f"basis shape {basis.shape} != ({d}, {d})")
    if len(cfg.names) != n:
        raise ValueError(f"{len(cfg.names)} names for {n} particles")
    if any(len(nm) != NAME_BYTES for nm in cfg.names):
        raise ValueError(f"each name must be exactly {NAME_BYTES} bytes")
    recs = np.empty(n, dtype=_record_dtype(d))
    recs["x"] = rel
    recs["name"] = np.frombuffer(b"".join(cfg.names), dtype="V4")
    head = struct.pack("<Hd", d, float(cfg.cell_size))
    return b"".join((head, basis.astype("<f8").tobytes(), struct.pack("<i", n), recs.tobytes()))


def read_configpack(prefix: Path, indices: Optional[Sequence[int]] = None) -> List[PackedConfig]:
    """Read configurations ``indices`` (all when None; order and repeats kept).

    ``FileNotFoundError`` when either file is missing; ``ValueError`` on
    truncated or malformed files or an index out of range.
    """
    pack_path, index_path = _files(Path(prefix))
    if not (pack_path.is_file() and index_path.is_file()):
        raise FileNotFoundError(f"need both {pack_path} and {index_path} (pack exists: "
                                f"{pack_path.is_file()}, index exists: {index_path.is_file()})")  # fmt: skip
    offs = _offsets(index_path)
    sel = list(range(offs.size)) if indices is None else [int(i) for i in indices]
    if any(i < 0 or i >= offs.size for i in sel):
        raise ValueError(f"config index outside [0, {offs.size})")
    if not sel:
        return []
    if os.path.getsize(pack_path) == 0:
        raise ValueError(f"empty pack for {offs.size} configs: {pack_path}")
    data = memoryview(pack_path.read_bytes())
    return [_decode(data, int(offs[i])) for i in sel]


def write_configpack(prefix: Path, configs: Sequence[PackedConfig]) -> None:
    """Write ``configs`` as ``prefix.ConfigPack`` + ``prefix.ConfigPackIndex``.

    ``FileNotFoundError`` if the parent directory is missing; ``ValueError``
    or ``TypeError`` on an empty sequence, bad shapes, names or dtypes.
    """
    prefix = Path(prefix)
    if not prefix.parent.is_dir():
        raise FileNotFoundError(f"missing parent directory: {prefix.parent}")
    if len(configs) == 0:
        raise ValueError("refusing to write an empty configuration sequence")
    blobs = [_encode(c) for c in configs]
    offs = np.zeros(len(blobs) + 1, dtype="<i8")
    offs[0] = len(blobs)
    offs[2:] = np.cumsum([len(b) for b in blobs[:-1]], dtype=np.int64)
    pack_path, index_path = _files(prefix)
    pack_path.write_bytes(b"".join(blobs))
    index_path.write_bytes(offs.tobytes())


def stack_fractional(configs: Sequence[PackedConfig]) -> Tuple[np.ndarray, np.ndarray]:
    """((B, N, d) fractional positions, (d, d) unit-volume basis) of a pack.

    The unit basis is ``basis / det(basis)^(1/d)``, required equal across the
    configurations (relative 1e-12). ``ValueError`` on an empty sequence,
    mixed shapes, a non-positive determinant or differing bases;
    ``TypeError`` on non-float64 arrays.
    """
    if len(configs) == 0:
        raise ValueError("no configurations to stack")
    shape = np.asarray(configs[0].relative).shape
    units = []
    for c in configs:
        rel, basis = np.asarray(c.relative), np.asarray(c.basis)
        if rel.dtype != np.float64 or basis.dtype != np.float64:
            raise TypeError("positions and basis must be float64")
        if rel.shape != shape:
            raise ValueError(f"mixed shapes {rel.shape} and {shape}")
        d = shape[1]
        if basis.shape != (d, d):
            raise ValueError(f"basis shape {basis.shape} != ({d}, {d})")
        det = float(np.linalg.det(basis))
        if not det > 0.0:
            raise ValueError(f"non-positive basis determinant {det}")
        units.append(basis / det ** (1.0 / d))
    for u in units[1:]:
        if not np.allclose(u, units[0], rtol=_UNIT_RTOL, atol=_UNIT_RTOL):
            raise ValueError("bases differ across configurations")
    return np.stack([np.asarray(c.relative) for c in configs]), units[0]
