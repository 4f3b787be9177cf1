"""Fail-fast GPU guard (``src/xla_cco/_device.py:137-142`` of the reference).

``require_gpu`` raises ``RuntimeError`` naming the most likely cause when no
CUDA device can be used, so a job never silently runs somewhere else (this
build has no CPU path at all):

- ``CUDA_VISIBLE_DEVICES`` set to an empty or invalid list: no device exposed
  to the process (a scheduler allocation without a GPU);
- ``libcco.so`` not built: run ``python xla-cco_b200/build.py``;
- otherwise: the CUDA driver reports no usable device.
"""

from __future__ import annotations

import os
from typing import Mapping, Optional

from xla_cco import _native


def classify_failure(n_devices: int, env: Mapping[str, str], lib_error: Optional[str]) -> Optional[str]:
    """The likely cause when ``n_devices`` is 0 (None when a device is visible)."""
    if lib_error is not None:
        return f"the CUDA library cannot be loaded: {lib_error}"
    if n_devices > 0:
        return None
    vis = env.get("CUDA_VISIBLE_DEVICES")
    if vis is not None and vis.strip() in ("", "-1", "none", "NoDevFiles"):
        return (f"no GPU exposed to this process (CUDA_VISIBLE_DEVICES={vis!r}); request a GPU "
                "from the scheduler or unset the variable")  # fmt: skip
    return "no CUDA device visible to the driver, and this build has no CPU path"


def require_gpu() -> None:
    """Raise RuntimeError naming the likely cause unless a GPU is visible."""
    lib_error = None
    n = 0
    try:
        n = _native.device_count()
    except RuntimeError as exc:   # libcco.so missing
        lib_error = str(exc)
    cause = classify_failure(n, os.environ, lib_error)
    if cause is not None:
        raise RuntimeError(cause)
