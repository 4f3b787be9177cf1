"""Generate tests/golden/io_golden.{npz,json} from the reference checkout.

    python tests/golden/make_io_golden.py --ref <reference checkout>   (or XLA_CCO_REFERENCE=<path>)

Covers the callers either side of the relaxation path: the ConfigPack format,
the C++ function-table writer, the isotropic S(k) k-set and binning, and the
pair-statistics oracle. Imported from the reference by file path (NumPy-only
code; its package __init__ needs JAX):

* ``src/xla_cco/io/configpack.py`` and ``src/xla_cco/io/tables.py``;
* ``src/xla_cco/kvectors.py`` and ``tests/oracle.py``;
* the functions ``_isotropic_kset`` and ``_bin_moments`` of
  ``src/xla_cco/analysis/structure.py``, extracted with ``ast`` (the module
  imports JAX at the top) and executed with the reference's
  ``enumerate_kvectors``.

The bundled input packs ``tests/data/inputs/*`` are decoded with the
reference reader; their decoded fields and the SHA-256 of the original files
are stored, not the files. Tests never read the reference checkout.
"""

from __future__ import annotations

import argparse
import os
import ast
import hashlib
import importlib.util
import json
import math
import tempfile
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
SHEARED_2D = np.array([[1.3, 0.0], [0.4, 0.9]])


def _load(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _extract(path: Path, names: list[str], ns: dict) -> dict:
    tree = ast.parse(path.read_text())
    fns = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    for fn in fns:
        fn.returns = None
        for a in fn.args.args:
            a.annotation = None
    exec(compile(ast.Module(body=fns, type_ignores=[]), str(path), "exec"), ns)
    return {n: ns[n] for n in names}


def _names(n: int, seed: int) -> tuple:
    rng = np.random.default_rng(seed)
    return tuple(bytes(rng.integers(0, 256, size=4, dtype=np.uint8)) for _ in range(n))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("XLA_CCO_REFERENCE"),
                    required="XLA_CCO_REFERENCE" not in os.environ,
                    help="the reference checkout (default: $XLA_CCO_REFERENCE)")
    ref = Path(ap.parse_args().ref)
    cp = _load(ref / "src/xla_cco/io/configpack.py", "ref_configpack")
    tb = _load(ref / "src/xla_cco/io/tables.py", "ref_tables")
    kv = _load(ref / "src/xla_cco/kvectors.py", "ref_kvectors")
    orc = _load(ref / "tests/oracle.py", "ref_oracle")
    st = _extract(ref / "src/xla_cco/analysis/structure.py", ["_isotropic_kset", "_bin_moments"],
                  {"np": np, "math": math, "enumerate_kvectors": kv.enumerate_kvectors,
                   "Tuple": tuple})  # fmt: skip
    arrays: dict[str, np.ndarray] = {}
    meta: dict = {"packs": [], "inputs": [], "tables": [], "iso": [], "bins": [], "pairs": [],
                  "sk": []}  # fmt: skip

    # ---- ConfigPack written by the reference writer (seeded configurations)
    groups = [
        [(5, 2, 1.5, 1.0), (3, 3, 2.0, 0.7)],
        [(10, 3, 1.0, 1.0), (4, 2, 1.5, 2.0), (1, 1, 3.0, 1.0)],
        [(0, 2, 1.0, 1.0), (7, 4, 1.0, 1.0), (64, 2, 8.0, 8.0)],
    ]
    with tempfile.TemporaryDirectory() as tmp:
        for g, group in enumerate(groups):
            rng = np.random.default_rng(100 + g)
            cfgs = []
            for i, (n, d, scale, cell) in enumerate(group):
                basis = np.eye(d) * scale + np.triu(rng.uniform(-0.3, 0.3, size=(d, d)), 1)
                cfgs.append(cp.PackedConfig(basis, rng.uniform(-1.0, 2.0, size=(n, d)), cell,
                                            _names(n, 1000 * g + i)))  # fmt: skip
            prefix = Path(tmp) / f"g{g}"
            cp.write_configpack(prefix, cfgs)
            pack = Path(str(prefix) + cp.PACK_SUFFIX).read_bytes()
            index = Path(str(prefix) + cp.INDEX_SUFFIX).read_bytes()
            arrays[f"pack{g}_bytes"] = np.frombuffer(pack, dtype=np.uint8)
            arrays[f"pack{g}_index"] = np.frombuffer(index, dtype=np.uint8)
            for i, c in enumerate(cp.read_configpack(prefix)):
                arrays[f"pack{g}_{i}_basis"] = c.basis
                arrays[f"pack{g}_{i}_rel"] = c.relative
                arrays[f"pack{g}_{i}_names"] = np.frombuffer(b"".join(c.names) or b"", np.uint8)
            meta["packs"].append({"group": g, "count": len(cfgs),
                                  "cells": [c.cell_size for c in cfgs]})  # fmt: skip

    # ---- bundled input packs: decoded fields + file hashes
    for pack in sorted((ref / "tests/data/inputs").glob("*.ConfigPack")):
        prefix = pack.with_suffix("")
        cfgs = cp.read_configpack(prefix)
        key = prefix.name
        s, unit = cp.stack_fractional(cfgs)
        arrays[f"in_{key}_s"] = s
        arrays[f"in_{key}_unit"] = unit
        arrays[f"in_{key}_bases"] = np.stack([c.basis for c in cfgs])
        arrays[f"in_{key}_names"] = np.frombuffer(b"".join(b"".join(c.names) for c in cfgs), np.uint8)
        meta["inputs"].append({
            "name": key, "count": len(cfgs), "cells": [c.cell_size for c in cfgs],
            "pack_sha256": hashlib.sha256(pack.read_bytes()).hexdigest(),
            "index_sha256": hashlib.sha256(Path(str(prefix) + cp.INDEX_SUFFIX).read_bytes()).hexdigest(),
        })  # fmt: skip

    # ---- function tables
    cases = [
        [np.array([1.5, -2.0]), np.array([0.0, 1e-22])],
        [np.array([1.3536712390e00]), np.array([2.4540768640e-22]), np.array([0.0]),
         np.array([1.1926785651e-23])],
        [np.array([np.nan, -np.nan, -0.0, 5e-324, 1.7976931348623157e308, 123456.789e-300])],
        [np.linspace(-3.0, 7.0, 11), np.geomspace(1e-30, 1e30, 11), np.arange(11.0) / 3.0],
    ]
    with tempfile.TemporaryDirectory() as tmp:
        for t, cols in enumerate(cases):
            path = Path(tmp) / f"t{t}.txt"
            tb.write_function_table(path, cols)
            for j, c in enumerate(cols):
                arrays[f"table{t}_col{j}"] = c
            meta["tables"].append({"case": t, "n_cols": len(cols), "text": path.read_text()})

    # ---- isotropic S(k) k-set (C++ GetKs order)
    iso = [
        ("d1_2.7", np.array([[2.7]]), 5.0, 30.0),
        ("sheared2", SHEARED_2D, 6.0, 14.0),
        ("cubic3_1.9", np.eye(3) * 1.9, 4.0, 9.0),
        ("d1_20", np.array([[20.0]]), 5.0, 8.0),
        ("sheared2x3", SHEARED_2D * 3.0, 3.0, 10.0),
        ("cubic3_6", np.eye(3) * 6.0, 2.5, 6.0),
        ("eq1", np.eye(1) * 2.0 * math.pi, 3.0, 5.0),
        ("eq2", np.eye(2) * 2.0 * math.pi, 3.0, 5.0),
        ("eq3", np.eye(3) * 2.0 * math.pi, 3.0, 5.0),
        ("cli_d2_n64", np.eye(2) * 8.0, 5.0, 400.0),
        ("cli_d3_n100", np.eye(3) * 100.0 ** (1.0 / 3.0), 5.0, 400.0),
        ("cli_d1_n50", np.eye(1) * 50.0, 5.0, 400.0),
    ]
    for name, basis, kd, km in iso:
        nv, k2 = st["_isotropic_kset"](basis, kd, km)
        arrays[f"iso_{name}_basis"] = basis
        arrays[f"iso_{name}_n"] = nv
        arrays[f"iso_{name}_ksq"] = k2
        meta["iso"].append({"name": name, "k_dir": kd, "k_max": km, "m": int(nv.shape[0])})

    # ---- C++ binning of per-k moments
    for b, (m, n_cfg, width) in enumerate([(200, 3, 0.05), (57, 1, 0.01), (1000, 7, 0.5)]):
        rng = np.random.default_rng(300 + b)
        k = np.sort(rng.uniform(0.1, 5.0, size=m))
        sm = rng.uniform(0.0, 2.0, size=m)
        s2 = sm * sm * rng.uniform(0.8, 1.6, size=m)
        out = st["_bin_moments"](k, sm, s2, n_cfg, width)
        for j, name in enumerate(("k", "s", "s2")):
            arrays[f"bins{b}_in_{name}"] = (k, sm, s2)[j]
        for j in range(4):
            arrays[f"bins{b}_out{j}"] = out[j]
        meta["bins"].append({"case": b, "n_cfg": n_cfg, "width": width})
    k = np.full(3, 0.1)
    out = st["_bin_moments"](k, np.ones(3), np.full(3, 0.5), 1, 0.01)
    meta["bins_negative_variance"] = [float.hex(float(v[0])) if v[0] == v[0] else "nan" for v in out]

    # ---- pair statistics (reference oracle, 3^d image scan)
    pairs = [("sheared2_16", SHEARED_2D, 16, 5), ("cubic3_12", np.eye(3) * 2.3, 12, 6),
             ("d1_9", np.array([[4.0]]), 9, 7), ("cubic2_30", np.eye(2) * 5.0, 30, 8)]
    for name, basis, n, seed in pairs:
        s = np.random.default_rng(seed).uniform(size=(n, basis.shape[0]))
        arrays[f"pairs_{name}_s"] = s
        arrays[f"pairs_{name}_basis"] = basis
        arrays[f"pairs_{name}_nn"] = orc.nearest_neighbor_distances(s, basis)
        arrays[f"pairs_{name}_dist"] = orc.pair_distances(s, basis)
        meta["pairs"].append({"name": name})

    # ---- structure factor (reference oracle direct sum)
    for name, n, d, seed in [("sk2", 20, 2, 9), ("sk3", 11, 3, 10)]:
        rng = np.random.default_rng(seed)
        s = rng.uniform(size=(n, d))
        nv = rng.integers(-4, 5, size=(15, d)).astype(np.float64)
        nv = nv[np.any(nv != 0, axis=1)]
        nv = np.unique(nv, axis=0)
        arrays[f"sk_{name}_s"] = s
        arrays[f"sk_{name}_n"] = nv
        arrays[f"sk_{name}_out"] = orc.structure_factor(s, nv)
        meta["sk"].append({"name": name})

    np.savez_compressed(OUT / "io_golden.npz", **arrays)
    (OUT / "io_golden.json").write_text(json.dumps(meta, indent=1) + "\n")
    print(f"wrote {len(arrays)} arrays")


if __name__ == "__main__":
    main()
