"""Generate tests/golden/relax_golden.{npz,json}: the CPU oracle's relaxations
of the two plain FP64 workloads, run to completion on their exact seeds.

    python tests/golden/make_relax_golden.py [--threads T] [--only cfg1|cfg2]

Workloads (the reference's own conventions: ``default_rng(seed).uniform``
positions, cubic unit-density box, packing fraction 0.05, K1 = 0):

* descent_d3_n100: d = 3, N = 100, chi = 0.05 (M = 13), batch 5, seed 0,
  DescentSettings(grow=2.0, max_evals=200_000, energy_tol=9.99999968e-21) -
  the reference README's relax call with the ground-state driver's default
  tolerance (README.md:78, src/xla_cco/cli/relax.py:84);
* lbfgs_d2_n1000: d = 2, N = 1000, chi = 0.40 (M = 802), batch 256, seed 0,
  LBFGSSettings(energy_tol=1e-20).

The oracle (oracle/cco_oracle.c, OpenMP over lanes) restates the reference's
trig energy, its descent loop and the L-BFGS schedule; it is pinned against
the reference's golden data elsewhere (tests/test_oracle.py). Stored per lane:
final energy, gradient norm, status, evaluation and iteration counts, and the
success mask energy < tol; the descent workload also keeps final positions
(5 x 100 x 3). The k-set comes from xla_cco.kvectors, which reproduces the
reference's enumeration bit for bit (tests/test_kvectors.py). The cfg2 run
takes about 4000 CPU-seconds; the fixtures are committed and the tests read
only them.
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
ROOT = OUT.parents[1]
for _p in (ROOT / "xla-cco_b200", ROOT / "oracle"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

DESCENT_TOL = 9.99999968e-21
WORKLOADS = {
    "descent_d3_n100": dict(n=100, d=3, chi=0.05, batch=5, seed=0, method="descent"),
    "lbfgs_d2_n1000": dict(n=1000, d=2, chi=0.40, batch=256, seed=0, method="lbfgs"),
}


def workload_inputs(name: str):
    """(s0, kset n (M, d) int64, weights, volume, settings, tol) of a workload."""
    from xla_cco import DescentSettings, LBFGSSettings, cubic_box, enumerate_kvectors
    from xla_cco import k_outer_from_ka, ka_from_chi

    w = WORKLOADS[name]
    box = cubic_box(w["n"], w["d"])
    ks = enumerate_kvectors(box.basis, 0.0,
                            k_outer_from_ka(ka_from_chi(w["chi"], 0.05, w["d"]), 0.05, w["d"]))
    s0 = np.random.default_rng(w["seed"]).uniform(size=(w["batch"], w["n"], w["d"]))
    if w["method"] == "descent":
        st = DescentSettings(grow=2.0, max_evals=200_000, energy_tol=DESCENT_TOL)
        tol = DESCENT_TOL
    else:
        st = LBFGSSettings(energy_tol=1e-20)
        tol = 1e-20
    return s0, ks.n, ks.weights, float(box.volume), st, tol


def main() -> None:
    import oracle

    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--only", choices=sorted(WORKLOADS), default=None)
    args = ap.parse_args()
    npz_path, json_path = OUT / "relax_golden.npz", OUT / "relax_golden.json"
    arrays = dict(np.load(npz_path)) if npz_path.exists() else {}
    meta = json.loads(json_path.read_text()) if json_path.exists() else {}
    for name, w in WORKLOADS.items():
        if args.only and name != args.only:
            continue
        s0, n, wts, vol, st, tol = workload_inputs(name)
        t0 = time.perf_counter()
        out = oracle.relax_batch(w["method"], s0, n, wts, vol, st, threads=args.threads)
        dt = time.perf_counter() - t0
        for k in ("energy", "grad_norm", "status", "n_evals", "n_iters"):
            arrays[f"{name}/{k}"] = np.asarray(out[k])
        arrays[f"{name}/success"] = np.asarray(out["energy"] < tol)
        if w["method"] == "descent":
            arrays[f"{name}/s"] = np.asarray(out["s"])
        meta[name] = dict(w, m=int(n.shape[0]), tol=tol, cpu_seconds=round(dt, 1),
                          threads=args.threads or oracle.max_threads(),
                          successes=int((out["energy"] < tol).sum()))  # fmt: skip
        print(name, meta[name], flush=True)
    np.savez_compressed(npz_path, **arrays)
    json_path.write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()
