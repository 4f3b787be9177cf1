"""Function tables in the C++ text layout (``WriteFunction``).

Mirrors ``src/xla_cco/io/tables.py:36-69`` of the reference: one line per
row, four fields (the C++ MaxDimension), each ``%1.10e`` followed by a TAB,
then a newline; missing columns are zeros. NaN prints as glibc does
(``nan`` / ``-nan`` by sign bit); infinities are refused.
"""

from __future__ import annotations

from pathlib import Path
from typing import Sequence

import numpy as np

N_FIELDS = 4


def _field(v: float) -> str:
    if v != v:
        return "-nan" if np.signbit(v) else "nan"
    return "%1.10e" % v


def write_function_table(path: Path, columns: Sequence[np.ndarray]) -> None:
    """Write 1 to 4 equal-length 1-D columns; ``ValueError`` otherwise or on inf."""
    if not 1 <= len(columns) <= N_FIELDS:
        raise ValueError(f"need 1..{N_FIELDS} columns, got {len(columns)}")
    cols = [np.asarray(c, dtype=np.float64) for c in columns]
    if any(c.ndim != 1 for c in cols):
        raise ValueError("columns must be 1-D")
    rows = cols[0].size
    if any(c.size != rows for c in cols):
        raise ValueError("columns have unequal lengths")
    table = np.zeros((rows, N_FIELDS))
    for j, c in enumerate(cols):
        table[:, j] = c
    if np.isinf(table).any():
        raise ValueError("infinite value in table")
    lines = ["".join(_field(v) + "\t" for v in row) + "\n" for row in table.tolist()]
    Path(path).write_bytes("".join(lines).encode("ascii"))
