"""Generate the golden fixtures in tests/golden/ from the reference checkout.

    python tests/golden/make_golden.py --ref <reference checkout>   (or XLA_CCO_REFERENCE=<path>)

Only the reference's NumPy-only modules are imported (by file path, without
its package __init__, which needs JAX): src/xla_cco/kvectors.py,
tests/oracle.py, plus its data files tests/data/md_cxx_*.{json,npz}, and the
function ``_cpp_descent`` of tests/unit/test_descent.py (the test's verbatim
transcription of the C++ descent loop), extracted with ``ast`` and executed
against the reference oracle. Output: golden.npz + golden.json. The fixtures
are committed; tests never read the reference checkout.
"""

from __future__ import annotations

import argparse
import os
import ast
import importlib.util
import json
import math
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def _load(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _cpp_descent_fn(ref: Path, oracle_mod):
    src = (ref / "tests/unit/test_descent.py").read_text()
    tree = ast.parse(src)
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "_cpp_descent")
    mod = ast.Module(body=[fn], type_ignores=[])
    ns = {"np": np, "oracle": oracle_mod, "Any": object, "List": list, "Tuple": tuple}
    exec(compile(mod, "test_descent._cpp_descent", "exec"), ns)
    return ns["_cpp_descent"]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("XLA_CCO_REFERENCE"),
                    required="XLA_CCO_REFERENCE" not in os.environ,
                    help="the reference checkout (default: $XLA_CCO_REFERENCE)")
    ref = Path(ap.parse_args().ref)
    kv = _load(ref / "src/xla_cco/kvectors.py", "ref_kvectors")
    orc = _load(ref / "tests/oracle.py", "ref_oracle")
    arrays: dict[str, np.ndarray] = {}
    meta: dict = {"kset_cases": [], "scalars": {}, "energy_cases": [], "descent_cases": []}

    # ---- chi / cutoff conversions (bit patterns)
    sc = meta["scalars"]
    for d in (1, 2, 3, 4, 5):
        sc[f"unit_ball_volume_{d}"] = float.hex(kv.unit_ball_volume(d))
    for chi, d in [(0.05, 3), (0.40, 2), (0.45, 3), (0.49, 1), (0.10, 2), (0.25, 2), (0.35, 3)]:
        ka = kv.ka_from_chi(chi, 0.05, d)
        sc[f"ka_{chi}_{d}"] = float.hex(ka)
        sc[f"k2_{chi}_{d}"] = float.hex(kv.k_outer_from_ka(ka, 0.05, d))
    sc["chi_13_100_3"] = float.hex(kv.chi_from_count(13, 100, 3))

    # ---- k-sets: benchmark boxes, C++ MD box, sheared boxes, +-1 ulp shells
    cases = []
    for n, d, chi in [(100, 3, 0.05), (1000, 2, 0.40), (4000, 3, 0.45), (8000, 1, 0.49),
                      (200, 1, 0.05), (8000, 3, 0.49), (20000, 3, 0.45), (20000, 2, 0.45),
                      (100, 2, 0.10), (64, 2, 0.25), (100, 3, 0.35), (12, 2, None),
                      (16, 2, None)]:  # fmt: skip
        basis = float(n) ** (1.0 / d) * np.eye(d)
        k2 = 4.0 if chi is None else kv.k_outer_from_ka(kv.ka_from_chi(chi, 0.05, d), 0.05, d)
        cases.append((f"cubic_n{n}_d{d}_chi{chi}", basis, 0.0, k2))
    md = json.loads((ref / "tests/data/md_cxx_reference.json").read_text())
    cases.append(("md_cxx", np.array(md["basis"], dtype=np.float64), 0.0, float(md["K"])))
    cases.append(("sheared3", np.array([[1.0, 0, 0], [8.0, 1, 0], [-6.0, 7, 1]]), 0.0, 9.0))
    base = np.array([[1.0, 0, 0], [0.9, 1, 0], [0.7, 0.8, 1]])
    for k2 in (3.0, 5.0, 8.0):
        cases.append((f"scaled_sheared_{k2}", 4.0 * base, 0.0, k2))
    cases.append(("sheared2_annulus", np.array([[2.0, 0.0], [0.7, 1.5]]), 0.5, 6.0))
    for side in (1.0, 2.0, 3.7):
        for d in (1, 2, 3):
            basis = side * np.eye(d)
            unit = float(orc.reciprocal_basis(basis)[0, 0])
            up, down = float(np.nextafter(unit, np.inf)), float(np.nextafter(unit, 0.0))
            cases.append((f"ulp_out_eq_{side}_{d}", basis, 0.0, unit))
            cases.append((f"ulp_out_up_{side}_{d}", basis, 0.0, up))
            cases.append((f"ulp_in_eq_{side}_{d}", basis, unit, 1.2 * unit))
            cases.append((f"ulp_in_dn_{side}_{d}", basis, down, 1.2 * unit))
    for i, (name, basis, k1, k2) in enumerate(cases):
        ks = kv.enumerate_kvectors(basis, k1, k2)
        arrays[f"kset{i}_basis"] = basis
        arrays[f"kset{i}_n"] = ks.n
        arrays[f"kset{i}_k"] = ks.k
        arrays[f"kset{i}_ksq"] = ks.k_sq
        meta["kset_cases"].append({"i": i, "name": name, "k_inner": float.hex(float(k1)),
                                   "k_outer": float.hex(float(k2)), "M": int(ks.n.shape[0])})  # fmt: skip

    # ---- energies and C++ forces from the reference oracle (small systems)
    ecases = [(0, 12, 2, 4.0), (3, 12, 2, 4.0), (5, 6, 2, 4.0), (4, 12, 2, 12.0),
              (7, 20, 2, 4.0), (11, 9, 1, 9.0), (12, 10, 3, 3.2), (1, 50, 2, 12.0),
              (2, 30, 3, 4.0), (9, 40, 1, 30.0)]  # fmt: skip
    for i, (seed, n, d, k2) in enumerate(ecases):
        basis = float(n) ** (1.0 / d) * np.eye(d)
        ks = kv.enumerate_kvectors(basis, 0.0, k2)
        s = np.random.default_rng(seed).uniform(size=(n, d))
        vol = float(abs(np.linalg.det(basis)))
        e = orc.energy(s, ks.n, ks.weights, vol)
        f = orc.cartesian_forces(s, ks.n, ks.weights, basis, vol)
        arrays[f"energy{i}_s"] = s
        arrays[f"energy{i}_n"] = ks.n
        arrays[f"energy{i}_basis"] = basis
        arrays[f"energy{i}_forces"] = f
        meta["energy_cases"].append({"i": i, "seed": seed, "n": n, "d": d, "k_outer": k2,
                                     "volume": vol, "phi": e})  # fmt: skip

    # ---- C++ golden energies (md_cxx samples)
    with np.load(ref / "tests/data/md_cxx_samples.npz") as z:
        arrays["cxx_s"] = np.asarray(z["s"])
        arrays["cxx_basis"] = np.asarray(z["basis"])
        seeds, samples = np.asarray(z["seed"]), np.asarray(z["sample"])
    runs = {r["seed"]: r for r in md["runs"]}
    arrays["cxx_phi"] = np.array([runs[int(sd)]["phi_cpp"][int(k)] for sd, k in zip(seeds, samples)])
    meta["cxx"] = {"K": md["K"], "K_hex": md["K_hex"], "M": md["M"], "N": md["N"], "d": md["d"]}

    # ---- descent vs the reference test's transcription of the C++ loop
    cpp_descent = _cpp_descent_fn(ref, orc)
    for i, grow in enumerate((1.0, 2.0)):
        n, d, iters, step0 = 16, 2, 100, 3e-2
        basis = float(n) ** (1.0 / d) * np.eye(d)
        ks = kv.enumerate_kvectors(basis, 0.0, 4.0)
        s0 = np.random.default_rng(3).uniform(size=(n, d))
        xs, accepts, steps = cpp_descent(s0, ks, basis, float(abs(np.linalg.det(basis))),
                                         grow, iters, step0)  # fmt: skip
        arrays[f"descent{i}_s0"] = s0
        arrays[f"descent{i}_xs"] = np.array(xs)
        arrays[f"descent{i}_accepts"] = np.array(accepts)
        arrays[f"descent{i}_steps"] = np.array(steps)
        meta["descent_cases"].append({"i": i, "grow": grow, "n": n, "d": d, "iters": iters,
                                      "step0": step0, "k_outer": 4.0})  # fmt: skip

    np.savez_compressed(OUT / "golden.npz", **arrays)
    (OUT / "golden.json").write_text(json.dumps(meta, indent=1))
    print(f"wrote {len(arrays)} arrays, {len(meta['kset_cases'])} k-set cases")


if __name__ == "__main__":
    main()
