#!/usr/bin/env python3
"""Benchmark: batched L-BFGS relaxation to Phi < 1e-20 on B200.

Workload (one "step"): relax 256 seeded uniform configurations, d = 2,
N = 1000, chi = 0.40 (half-space k-set M = 802), cubic unit-density box,
LBFGSSettings(energy_tol = 1e-20) with the default three-pass schedule and
memory 100, all float64. Metric: relaxations/s to Phi < 1e-20 (lanes that
reach the tolerance, per second of device time), with p50/p99 lane latency.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU runs (torchrun, one process per GPU) are independent replicas:
lanes are independent relaxations, so each rank relaxes its own seeded batch
with no data-path collective; NCCL carries only the barrier and the max over
ranks of the timed region.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for _p in (ROOT / "xla-cco_b200", ROOT / "oracle"):
    sys.path.insert(0, str(_p))

METRIC = "relaxations/s to Phi<1e-20 (batched L-BFGS, plain FP64)"
UNIT = "relaxations/s"
N_PART, DIM, CHI, PHI_PACK, BATCH, SEED = 1000, 2, 0.40, 0.05, 256, 0
TOL = 1e-20
F_PAIR = {1: 7, 2: 21, 3: 35}  # algorithmic FP64 flops per (k, particle) pair and evaluation


def workload():
    from xla_cco import cubic_box, enumerate_kvectors, k_outer_from_ka, ka_from_chi, make_stealthy_energy

    box = cubic_box(N_PART, DIM)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(CHI, PHI_PACK, DIM), PHI_PACK, DIM))
    return box, ks, make_stealthy_energy(box, ks)


def oracle_inputs():
    """(basis, volume, k-set n) of the headline workload built by the oracle
    alone: its own cutoff formula and brute-force half-space scan in the
    reference's order (the same rows, bit for bit, as the product's
    enumeration). The CPU arms import nothing from the product package."""
    import oracle

    basis = float(N_PART) ** (1.0 / DIM) * np.eye(DIM)
    n = oracle.sorted_kset(basis, 0.0, oracle.k_outer_for_chi(CHI, PHI_PACK, DIM))
    return basis, float(abs(np.linalg.det(basis))), n


def config_dict(m: int, extra=None):
    c = {
        "workload": f"lbfgs_relax_d{DIM}_n{N_PART}_chi{CHI}_m{m}_b{BATCH}",
        "d": DIM, "n_particles": N_PART, "chi": CHI, "m_kvectors": int(m),
        "batch": BATCH, "energy_tol": TOL, "minimizer": "L-BFGS m=100, rescales 1e4/1/1e-2",
        "seeds": "default_rng(seed + rank).uniform((B, N, d))",
        "l2": "inputs larger than L2: history 2*100*N*d*8 B per lane = 0.8 GB per step",
    }  # fmt: skip
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")  # fmt: skip

    def __init__(self, index: int) -> None:
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )  # fmt: skip
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi's own start-up (driver and NVML initialisation) takes the
        # driver for a moment; let it finish before the caller starts timing,
        # so the timed region sees the steady 200 ms polling only
        t0 = time.perf_counter()
        while not self.lines and time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.02)
        time.sleep(0.25)

    def _read(self) -> None:
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


# ------------------------------------------------------------------ CPU arm
def cpu_relax(s0: np.ndarray, lanes, threads: int) -> tuple[int, int, float]:
    """Relax the given lanes of s0 to completion with the oracle L-BFGS (the
    reference's three-pass schedule, energy_tol 1e-20), one lane after another,
    each evaluation spread over `threads` host threads. Returns (successes,
    evaluations, wall seconds)."""
    import oracle

    basis, vol, n = oracle_inputs()
    st = oracle.lbfgs_settings(energy_tol=TOL)
    lanes = list(lanes)
    t0 = time.perf_counter()
    out = oracle.relax_lanes("lbfgs", s0[lanes], n, np.ones(n.shape[0]), vol, st, threads=threads)
    dt = time.perf_counter() - t0
    return int((out["energy"] < TOL).sum()), int(out["n_evals"].sum()), dt


def cpu_sample(s0: np.ndarray, min_seconds: float = 10.0, max_lanes: int = 16) -> dict:
    """cpu_baseline: the oracle relaxes lanes 0, 1, ... of the same seeded
    batch to Phi < 1e-20 on all host threads until `min_seconds` have passed
    (at most `max_lanes`); value = completed relaxations / wall time."""
    import oracle

    threads = oracle.max_threads()
    succ = evals = 0
    wall = 0.0
    lane = 0
    while lane < min(max_lanes, s0.shape[0]) and (lane == 0 or wall < min_seconds):
        s, e, dt = cpu_relax(s0, [lane], threads)
        succ, evals, wall, lane = succ + s, evals + e, wall + dt, lane + 1
    return {
        "value": succ / wall, "unit": UNIT, "cores": threads, "kind": "port",
        "evals_per_s": evals / wall,
        "sample": (f"C oracle (direct-sum FP64 energy, L-BFGS three-pass schedule) relaxing lanes "
                   f"0..{lane - 1} of the seeded batch to Phi<1e-20, one after another, each "
                   f"evaluation on {threads} host threads: {succ}/{lane} relaxed, {evals} "
                   f"evaluations in {wall:.1f} s"),
    }  # fmt: skip


def run_reference(args) -> None:
    """The reference arm: the CPU restatement of the reference's path (the
    oracle; the reference's JAX package cannot be installed here) relaxing
    lanes of the same seeded batch to Phi < 1e-20. Step i relaxes lane i to
    completion on every host thread; value = completed relaxations / wall
    time of the timed steps. Imports nothing from the product package."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle

    threads = oracle.max_threads()
    _, _, n = oracle_inputs()
    s0 = np.random.default_rng(SEED).uniform(size=(BATCH, N_PART, DIM))
    for i in range(args.warmup):
        cpu_relax(s0, [i % BATCH], threads)
    succ = evals = 0
    wall = 0.0
    first = args.warmup % BATCH
    for i in range(args.steps):
        s, e, dt = cpu_relax(s0, [(args.warmup + i) % BATCH], threads)
        succ, evals, wall = succ + s, evals + e, wall + dt
    value = succ / wall
    cb = {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
          "evals_per_s": evals / wall,
          "sample": (f"C oracle relaxing lanes {first}..{(first + args.steps - 1) % BATCH} of the "
                     f"seeded batch to Phi<1e-20 (one lane per step, each evaluation on {threads} "
                     f"host threads): {succ}/{args.steps} relaxed, {evals} evaluations in "
                     f"{wall:.1f} s")}  # fmt: skip
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_dict(n.shape[0]),
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }  # fmt: skip
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ranks
def rank_totals(dist, t_ms: float, succ: int, device: str) -> tuple[float, int]:
    """(largest t_ms over the ranks, sum of succ over the ranks); unchanged
    for a single process (``dist`` None). Every rank must call it, in the same
    order as the other collectives."""
    if dist is None:
        return t_ms, succ
    import torch

    mx = torch.tensor([t_ms], dtype=torch.float64, device=device)
    sm = torch.tensor([float(succ)], dtype=torch.float64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), int(round(float(sm[0])))


# ------------------------------------------------------------------ device arm
def fp64_peak_tflops() -> float | None:
    import ctypes

    lib_path = ROOT / "xla-cco_b200" / "xla_cco" / "_lib" / "libcco_peaks.so"
    if not lib_path.exists():
        return None
    lib = ctypes.CDLL(str(lib_path))
    out = ctypes.c_double(0.0)
    best = 0.0
    for _ in range(3):
        if lib.cco_peak_fma(1, 148 * 8, 256, 2000, ctypes.byref(out)) == 0:
            best = max(best, out.value)
    return best or None


def run_device(args) -> None:
    import torch

    from xla_cco import LBFGSSettings, relax
    from xla_cco.minimize import relax_device

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    box, ks, energy = workload()
    settings = LBFGSSettings(energy_tol=TOL)
    s0 = np.random.default_rng(SEED + rank).uniform(size=(args.batch, N_PART, DIM))
    s_dev = torch.from_numpy(s0).cuda()
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        relax_device(energy, s_dev, settings)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    outs = []
    for _ in range(args.steps):
        outs.append(relax_device(energy, s_dev, settings))
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    succ = sum(int((o["energy"] < TOL).sum().item()) for o in outs)
    evals = np.concatenate([o["n_evals"].cpu().numpy() for o in outs])
    lat = np.concatenate([o["latency_ns"].cpu().numpy() for o in outs]) / 1e6
    launches = sum(o["launches"] for o in outs)
    ticks = sum(o["ticks"] for o in outs)
    t_max, succ = rank_totals(dist, ms, succ, "cuda")
    value = succ / (t_max / 1e3)

    # roofline of the evaluation kernels (pass 1 + reduce + pass 2) on this batch
    ev_n = 20
    for _ in range(3):
        energy.evaluate(s_dev)
    torch.cuda.synchronize()
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    for _ in range(ev_n):
        energy.evaluate(s_dev)
    r1.record(stream)
    torch.cuda.synchronize()
    eval_ms = r0.elapsed_time(r1) / ev_n
    m = int(ks.n.shape[0])
    flop = float(args.batch) * N_PART * m * F_PAIR[DIM]
    achieved = flop / (eval_ms * 1e-3) / 1e12
    peak = fp64_peak_tflops()
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("eval_bytes_per_launch")

    # end to end through the public API: pinned host in, host out, every step
    # (whole job: successes summed over the ranks, the slowest rank's wall time)
    pinned = torch.from_numpy(s0).pin_memory()
    h2d = pinned.numel() * 8
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    e2e_succ = 0
    for _ in range(args.steps):
        res = relax(energy, pinned, settings)
        e2e_succ += int((res.energy < TOL).sum())
    e2e_s = time.perf_counter() - t0
    barrier()
    e2e_ms, e2e_succ = rank_totals(dist, e2e_s * 1e3, e2e_succ, "cuda")
    d2h = args.batch * (N_PART * DIM * 8 + 8 * 5)
    e2e = {"value": e2e_succ / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h,
           "timing": "host wall clock around relax(numpy->numpy), max over ranks"}  # fmt: skip

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    epr = float(evals.mean())
    cb = None
    if not args.no_cpu_baseline:
        cb = cpu_sample(s0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(int(ks.n.shape[0]), {
            "parallelism": f"replicas x{world}",
            "success": f"{succ}/{args.batch * args.steps * world}",
            "p50_latency_ms": float(np.percentile(lat, 50)),
            "p99_latency_ms": float(np.percentile(lat, 99)),
            "evals_per_relax": epr, "ticks": ticks,
            "schedule": {"branches": outs[-1]["schedule"][0], "graph_ticks": outs[-1]["schedule"][1],
                         "overlap": outs[-1]["overlap"]},
            "evals_per_s": float(evals.sum()) / (ms / 1e3),
            "pair_evals_per_s": float(evals.sum()) * N_PART * m / (ms / 1e3),
        }),
        "roofline": {
            "kernel": "energy+force evaluation (pass1 + reduce + pass2), batch 256",
            "bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if peak else None, "traffic": traffic,
            "eval_ms": eval_ms,
            "peak_source": "measured FP64 FMA probe (libcco_peaks.so), this run",
            "algorithmic": f"{F_PAIR[DIM]} flop per (k, particle) pair x N M x batch",
        },
        "cpu_baseline": cb,
        "e2e": e2e,
        "clocks": clocks,
        "gpu_launches": launches,
    }  # fmt: skip
    if world == 1 and not args.no_target:
        line["target"] = target_comparison()
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def target_comparison() -> dict:
    """The north-star comparison on the 512-instance mixed-size ensemble (N
    log-uniform in [200, 8000], d in {1, 2, 3}, chi in [0.05, 0.49], seed 0):
    the plain FP64 drop-in (one relax call per instance, every instance,
    sequential) against the batched device run and the served mixed-precision
    form, with success-mask equality and latency percentiles. Device time for
    the drop-in and the batch, host wall clock for the served stream."""
    import torch

    from xla_cco import LBFGSSettings
    from xla_cco.minimize import relax_mixed_device
    from xla_cco.workloads import mixed_ensemble

    inst = mixed_ensemble(512, seed=SEED)
    for i in inst:
        i.energy.problem_handle(torch.cuda.current_device(), i.n)
    settings = LBFGSSettings(energy_tol=TOL)
    flat = torch.from_numpy(np.concatenate([i.s0.ravel() for i in inst])).cuda()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    out = relax_mixed_device([i.energy for i in inst], flat, [(i.n, i.d) for i in inst], settings)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ok = out["energy"].cpu().numpy() < TOL
    lat = out["latency_ns"].cpu().numpy() / 1e6
    plain = plain_dropin(inst, settings, 0)
    plain_mask = plain.pop("mask")
    served = served_mixed(inst, plain_mask)
    return {
        "workload": "mixed_lbfgs_512_n200-8000_d123_chi0.05-0.49",
        "plain_fp64_dropin": plain,
        "batched_fp64": {"value": float(ok.sum()) / (ms / 1e3), "unit": UNIT, "ms": ms,
                         "success": f"{int(ok.sum())}/{len(inst)}",
                         "mask_equals_plain_dropin": bool((ok == plain_mask).all()),
                         "p50_latency_ms": float(np.percentile(lat, 50)),
                         "p99_latency_ms": float(np.percentile(lat, 99))},
        "served_mixed_precision": served,
        "served_speedup_vs_plain_dropin": served["value"] / plain["value"] if plain["value"] else None,
        "batched_speedup_vs_plain_dropin": (float(ok.sum()) / (ms / 1e3)) / plain["value"]
        if plain["value"] else None,
    }  # fmt: skip


# ------------------------------------------------------------------ mixed batch
def _flops(evals, inst) -> float:
    return float(sum(float(e) * i.n * i.m * F_PAIR[i.d] for e, i in zip(evals, inst)))


def plain_dropin(inst, settings, sample: int) -> dict:
    """The reference's usage on a mixed ensemble: one relax call per instance
    (relax takes one energy, so instances of different N, d, chi cannot share
    a call). Times the first `sample` instances (0: all of them) one after
    another, after one untimed pass over the same instances."""
    import torch

    from xla_cco.minimize import relax_device

    sub = inst[:sample] if sample > 0 else inst
    dev = [torch.from_numpy(i.s0[None]).cuda() for i in sub]
    for i, x in zip(sub, dev):
        relax_device(i.energy, x, settings)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    outs = [relax_device(i.energy, x, settings) for i, x in zip(sub, dev)]
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    succ = sum(int((o["energy"] < TOL).sum().item()) for o in outs)
    ok = np.array([bool((o["energy"] < TOL).item()) for o in outs])
    return {"value": succ / (ms / 1e3), "unit": UNIT, "instances": len(sub), "success": succ,
            "ms": ms, "how": "relax(energy_i, s0_i[None]) per instance, sequential, same device",
            "mask": ok}  # fmt: skip


def served_mixed(inst, ok_plain) -> dict:
    """The whole ensemble through the serving pool with mixed precision, all
    requests submitted at once; success mask compared with the plain batch."""
    from xla_cco import LBFGSSettings
    from xla_cco.serve import RelaxServer

    st = LBFGSSettings(energy_tol=TOL, precision="mixed")
    with RelaxServer(st) as srv:
        t0 = time.perf_counter()
        tickets = [srv.submit(i.energy, i.s0) for i in inst]
        res = [srv.result(t) for t in tickets]
        wall = time.perf_counter() - t0
        stats = srv.stats()
    ok = np.array([r.energy < TOL for r in res])
    lat = np.array([r.latency_s for r in res]) * 1e3
    n32 = sum(r.n_evals_fp32 for r in res)
    ev = sum(r.n_evals for r in res)
    return {"value": float(ok.sum()) / wall, "unit": UNIT, "wall_s": wall,
            "success": f"{int(ok.sum())}/{len(inst)}",
            "success_mask_equals_plain_fp64": bool((ok == ok_plain).all()),
            "mask_differences": int((ok != ok_plain).sum()),
            "p50_latency_ms": float(np.percentile(lat, 50)),
            "p99_latency_ms": float(np.percentile(lat, 99)),
            "fp32_eval_fraction": n32 / max(ev, 1), "peak_lanes": stats.peak_lanes,
            "timing": "host wall clock from the first submission to the last result"}  # fmt: skip


def run_mixed(args) -> None:
    import torch

    from xla_cco import LBFGSSettings
    from xla_cco.minimize import relax_mixed_device
    from xla_cco.workloads import mixed_ensemble

    torch.cuda.set_device(0)
    inst = mixed_ensemble(args.mixed_count, seed=SEED)
    energies = [i.energy for i in inst]
    shapes = [(i.n, i.d) for i in inst]
    for i in inst:
        i.energy.problem_handle(0, i.n)
    flat = torch.from_numpy(np.concatenate([i.s0.ravel() for i in inst])).cuda()
    settings = LBFGSSettings(energy_tol=TOL)
    for _ in range(args.warmup):
        relax_mixed_device(energies, flat, shapes, settings)
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    outs = [relax_mixed_device(energies, flat, shapes, settings) for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    succ = sum(int((o["energy"] < TOL).sum().item()) for o in outs)
    evals = outs[-1]["n_evals"].cpu().numpy()
    lat = np.concatenate([o["latency_ns"].cpu().numpy() for o in outs]) / 1e6
    flops = _flops(evals, inst) * args.steps
    value = succ / (ms / 1e3)
    plain = plain_dropin(inst, settings, args.plain_sample)
    plain_mask = plain.pop("mask")
    batched_ok = outs[-1]["energy"].cpu().numpy() < TOL
    if plain_mask.size == batched_ok.size:
        plain["mask_equals_batched"] = bool((plain_mask == batched_ok).all())
    # the served mixed-precision form is judged against the plain drop-in's mask
    ref_mask = plain_mask if plain_mask.size == batched_ok.size else batched_ok
    served = served_mixed(inst, ref_mask) if args.served else None
    peak = fp64_peak_tflops()
    achieved = flops / (ms * 1e-3) / 1e12
    line = {
        "metric": "relaxations/s to Phi<1e-20 (mixed-size batch, one device run, plain FP64)",
        "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {
            "workload": f"mixed_lbfgs_{len(inst)}_n200-8000_d123_chi0.05-0.49",
            "instances": len(inst), "seeds": "xla_cco.workloads.mixed_ensemble(seed=0)",
            "success": f"{succ}/{len(inst) * args.steps}",
            "p50_latency_ms": float(np.percentile(lat, 50)),
            "p99_latency_ms": float(np.percentile(lat, 99)),
            "evals_per_relax": float(evals.mean()),
            "schedule": outs[-1]["schedule"], "ticks": outs[-1]["ticks"],
            "l2": "inputs larger than L2 (lane records of the whole ensemble)",
        },
        "plain_fp64_dropin": plain,
        "speedup_vs_plain_dropin": value / plain["value"] if plain["value"] else None,
        "served_mixed_precision": served,
        "served_speedup_vs_plain_dropin": (served["value"] / plain["value"]
                                           if served and plain["value"] else None),
        "roofline": {"kernel": "whole relaxation (evaluations + updates)", "bound": "fp64",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "algorithmic": "sum over lanes of evals x N M x flop/pair(d)"},  # fmt: skip
        "clocks": clocks,
        "gpu_launches": sum(o["launches"] for o in outs),
    }  # fmt: skip
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ descent (d3 N100)
DESCENT_TOL = 9.99999968e-21


def run_descent(args) -> None:
    """The reference README's relax call at the ground-state driver's default
    tolerance: d=3, N=100, chi=0.05 (M=13), batch 5 from seed 0,
    DescentSettings(grow=2.0, max_evals=200_000, energy_tol=9.99999968e-21).
    One step relaxes the 5 configurations; the oracle relaxes the same 5 on
    all host threads as the CPU baseline."""
    import oracle
    import torch

    from xla_cco import DescentSettings, cubic_box, enumerate_kvectors, k_outer_from_ka, ka_from_chi
    from xla_cco import make_stealthy_energy, relax
    from xla_cco.minimize import relax_device

    torch.cuda.set_device(0)
    n, d, chi, b = 100, 3, 0.05, 5
    box = cubic_box(n, d)
    ks = enumerate_kvectors(box.basis, 0.0, k_outer_from_ka(ka_from_chi(chi, PHI_PACK, d), PHI_PACK, d))
    en = make_stealthy_energy(box, ks)
    st = DescentSettings(grow=2.0, max_evals=200_000, energy_tol=DESCENT_TOL)
    s0 = np.random.default_rng(SEED).uniform(size=(b, n, d))
    s_dev = torch.from_numpy(s0).cuda()
    for _ in range(args.warmup):
        relax_device(en, s_dev, st)
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    outs = [relax_device(en, s_dev, st) for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    succ = sum(int((o["energy"] < DESCENT_TOL).sum().item()) for o in outs)
    iters = outs[-1]["n_iters"].cpu().numpy()
    lat = np.concatenate([o["latency_ns"].cpu().numpy() for o in outs]) / 1e6
    # end to end: host arrays in, host arrays out
    pinned = torch.from_numpy(s0).pin_memory()
    t0 = time.perf_counter()
    e2e_succ = 0
    for _ in range(args.steps):
        e2e_succ += int((relax(en, pinned, st).energy < DESCENT_TOL).sum())
    e2e_s = time.perf_counter() - t0
    cb = None
    if not args.no_cpu_baseline:
        threads = oracle.max_threads()
        reps, c_succ, wall = 0, 0, 0.0
        while reps == 0 or wall < 10.0:
            t0 = time.perf_counter()
            out = oracle.relax_batch("descent", s0, ks.n, ks.weights, box.volume, st, threads=threads)
            wall += time.perf_counter() - t0
            c_succ += int((out["energy"] < DESCENT_TOL).sum())
            reps += 1
        cb = {"value": c_succ / wall, "unit": UNIT, "cores": min(threads, b), "kind": "port",
              "sample": (f"C oracle descent on the same 5 configurations (one host thread per "
                         f"lane), {reps} repetitions: {c_succ}/{5 * reps} relaxed in {wall:.1f} s")}
    launches = sum(o["launches"] for o in outs)
    line = {
        "metric": "relaxations/s to Phi<9.99999968e-21 (batched adaptive descent, plain FP64)",
        "value": succ / (ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"descent_relax_d{d}_n{n}_chi{chi}_m{ks.n.shape[0]}_b{b}",
                   "settings": "DescentSettings(grow=2.0, max_evals=200000, energy_tol=9.99999968e-21)",
                   "success": f"{succ}/{b * args.steps}", "n_iters": iters.tolist(),
                   "p50_latency_ms": float(np.percentile(lat, 50)),
                   "p99_latency_ms": float(np.percentile(lat, 99)),
                   "l2": "latency-bound: 5 lanes of 1300 (k, particle) pairs"},
        "cpu_baseline": cb,
        "e2e": {"value": e2e_succ / e2e_s, "unit": UNIT, "h2d_bytes_per_step": s0.nbytes,
                "d2h_bytes_per_step": s0.nbytes + b * 8 * 5,
                "timing": "host wall clock around relax(numpy->numpy)"},
        "clocks": clocks, "gpu_launches": launches,
    }  # fmt: skip
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ precision
def run_precision(args) -> None:
    """d=3 N=4000 chi=0.45 batch 64: plain FP64 vs mixed precision, same seeds."""
    import oracle
    import torch

    from xla_cco import LBFGSSettings
    from xla_cco.minimize import relax_device
    from xla_cco.workloads import energy_for

    torch.cuda.set_device(0)
    n, d, chi, b = 4000, 3, 0.45, args.precision_batch
    en = energy_for(n, d, chi)
    box_vol = float(n)  # cubic unit-density box
    s0 = torch.from_numpy(np.random.default_rng(SEED).uniform(size=(b, n, d))).cuda()
    stream = torch.cuda.current_stream()
    out = {}
    sampler = ClockSampler(0)
    sampler.start()
    for name, prec in (("fp64", "fp64"), ("mixed", "mixed")):
        st = LBFGSSettings(energy_tol=TOL, precision=prec)
        for _ in range(args.warmup):
            relax_device(en, s0, st)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        runs = [relax_device(en, s0, st) for _ in range(args.steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        r = runs[-1]
        ok = (r["energy"] < TOL).cpu().numpy()
        out[name] = {"ms": ms / args.steps, "ok": ok, "energy": r["energy"].cpu().numpy(),
                     "s": r["s"].cpu().numpy(), "evals": r["n_evals"].cpu().numpy(),
                     "n32": r["n_evals_fp32"].cpu().numpy(),
                     "lat": r["latency_ns"].cpu().numpy() / 1e6}  # fmt: skip
    clocks = sampler.stop()
    # error of every mixed result against the FP64 oracle (direct sum, host threads)
    m = out["mixed"]
    ks_n = en.n_vectors[en._rows].astype(np.int64)
    w = en.weights[en._rows]
    e_ref, _ = oracle.energy_grad_batch(m["s"], ks_n, w, box_vol, threads=oracle.max_threads())
    errs = [abs(float(m["energy"][i]) - float(e_ref[i])) for i in range(b)]
    p, mx = out["fp64"], out["mixed"]
    line = {
        "metric": "relaxations/s to Phi<1e-20, mixed precision vs plain FP64 (same seeds)",
        "value": float(mx["ok"].sum()) / (mx["ms"] / 1e3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": mx["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic",
        "config": {
            "workload": f"lbfgs_relax_d3_n4000_chi0.45_m{en._rows.size}_b{b}_mixed_precision",
            "switch": "FP32 evaluations until Phi < 1e-6 N (or a stuck FP32 line search), then FP64",
            "success_mixed": f"{int(mx['ok'].sum())}/{b}", "success_fp64": f"{int(p['ok'].sum())}/{b}",
            "success_masks_identical": bool((mx["ok"] == p["ok"]).all()),
            "fp32_eval_fraction": float(mx["n32"].sum() / max(mx["evals"].sum(), 1)),
            "evals_per_relax_mixed": float(mx["evals"].mean()),
            "evals_per_relax_fp64": float(p["evals"].mean()),
            "max_abs_err_vs_fp64_oracle": float(max(errs)),
            "err_vs_fp64_oracle_per_result": [float(e) for e in errs],
            "p50_latency_ms": float(np.percentile(mx["lat"], 50)),
            "p99_latency_ms": float(np.percentile(mx["lat"], 99)),
        },
        "plain_fp64": {"value": float(p["ok"].sum()) / (p["ms"] / 1e3), "unit": UNIT,
                       "ms_per_step": p["ms"]},
        "speedup_vs_plain_fp64": (p["ms"] / mx["ms"]),
        "clocks": clocks,
    }  # fmt: skip
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ request stream
def run_serve(args) -> None:
    import torch

    from xla_cco import LBFGSSettings
    from xla_cco.serve import RelaxServer
    from xla_cco.workloads import request_stream

    torch.cuda.set_device(0)
    reqs = request_stream(args.serve_count, seed=SEED, rate=args.serve_rate)
    for r in reqs:
        r.energy.problem_handle(0, r.n)
    settings = LBFGSSettings(energy_tol=TOL, precision=args.serve_precision)
    sampler = ClockSampler(0)
    with RelaxServer(settings, hbm_budget_bytes=150 << 30, branches=args.serve_branches) as srv:
        # warm-up: a few requests through the pool before the stream starts
        for t in [srv.submit(r.energy, r.s0) for r in reqs[: args.warmup]]:
            srv.result(t)
        sampler.start()
        t0 = time.perf_counter()
        tickets = []
        for r in reqs:
            delay = t0 + r.arrival_s - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            tickets.append(srv.submit(r.energy, r.s0))
        results = [srv.result(t) for t in tickets]
        clocks = sampler.stop()
        st = srv.stats()
    first = min(x.submit_ns for x in results)
    last = max(x.done_ns for x in results)
    span = (last - first) * 1e-9
    succ = sum(1 for x in results if x.energy < TOL)
    lat = np.array([x.latency_s for x in results]) * 1e3
    queue = np.array([(x.admit_ns - x.submit_ns) * 1e-6 for x in results])
    dev = np.array([x.device_ns * 1e-6 for x in results])
    evals = np.array([x.n_evals for x in results])
    flops = _flops(evals, reqs)
    peak = fp64_peak_tflops()
    line = {
        "metric": "served relaxations/s to Phi<1e-20 + p50/p99 latency (Poisson stream)",
        "precision": args.serve_precision,
        "value": succ / span, "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": args.warmup,
        "ms_per_step": span * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {
            "workload": f"serve_lbfgs_{len(reqs)}req_{args.serve_rate:g}rps_n100-20000_d23_chi0.10-0.45",
            "requests": len(reqs), "rate_rps": args.serve_rate,
            "seeds": "xla_cco.workloads.request_stream(seed=0)", "hbm_budget_gb": 150,
            "success": f"{succ}/{len(reqs)}",
            "p50_latency_ms": float(np.percentile(lat, 50)),
            "p99_latency_ms": float(np.percentile(lat, 99)),
            "p50_queue_ms": float(np.percentile(queue, 50)),
            "p99_queue_ms": float(np.percentile(queue, 99)),
            "p50_device_ms": float(np.percentile(dev, 50)),
            "p99_device_ms": float(np.percentile(dev, 99)),
            "offered_span_s": reqs[-1].arrival_s,
            "server": {"peak_lanes": st.peak_lanes, "peak_gb": st.peak_bytes / 2**30,
                       "graphs": st.graphs, "ticks": st.ticks, "rebuilds": st.rebuilds},
        },
        "roofline": {"kernel": "whole served stream (evaluations + updates)", "bound": "fp64",
                     "achieved": flops / span / 1e12, "peak": peak, "unit": "TFLOP/s",
                     "frac": flops / span / 1e12 / peak if peak else None},
        "clocks": clocks,
    }  # fmt: skip
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ MD segments
def _md_host_sample(ks, basis, waves, r0, v0, n_steps: int) -> float:
    """Seconds per lane-step of the oracle chain (direct-sum forces and wave
    densities, NumPy on the host threads) over a short sample of one lane."""
    import oracle

    from xla_cco.dynamics import baoab_step, make_key

    inv = np.linalg.inv(basis)
    nv = ks.n.astype(np.float64)
    vol = float(abs(np.linalg.det(basis)))

    def force(r):
        s = r @ inv
        phi, g = oracle.energy_direct(s, nv, np.ones(nv.shape[0]), vol)
        re, im = oracle.density_direct(s, nv)
        return phi, -(g @ inv.T), re, im

    r, v, f, key = r0, v0, force(r0)[1], make_key(1)
    rho = np.zeros((waves.n_vectors.shape[0], 2))
    t0 = time.perf_counter()
    for _ in range(n_steps):
        key, r, v, out = baoab_step(key, r, v, f, force, 0.02, 1.0, 1e-3)
        f = out[1]
        rho, _ = oracle.md_observe(r, basis, waves.n_vectors, waves.kvec, waves.n_constrained, rho,
                                   True, True)  # fmt: skip
    return (time.perf_counter() - t0) / n_steps


def run_md(args) -> None:
    """MD segments (simulate) on the d=2 N=1000 chi=0.40 system: BAOAB lanes,
    tracked waves |k| < 1.5 K (constrained |k| < K), wind every 10 steps,
    200 snapshots and a rho trace every 20 steps (production recording)."""
    import torch

    from xla_cco.dynamics import MDSettings, init_state, make_key, make_waves, simulate

    torch.cuda.set_device(0)
    box, ks, energy = workload()
    basis = np.asarray(box.basis)
    from xla_cco import k_outer_from_ka, ka_from_chi

    k2 = k_outer_from_ka(ka_from_chi(CHI, PHI_PACK, DIM), PHI_PACK, DIM)
    waves = make_waves(basis, k2, 1.5 * k2)
    assert waves.n_constrained == ks.n.shape[0], "constrained waves are the energy's k-set"
    lanes, n_steps = args.md_lanes, args.md_steps
    st = MDSettings(dt=0.02, scheme="baoab", gamma=1.0, chunk_steps=n_steps, wind_every=10,
                    record_steps=tuple(range(n_steps // 200, n_steps + 1, max(n_steps // 200, 1)))[:200],
                    record_rho_every=20, max_rho_records=n_steps // 20, drift_tol=float("inf"))  # fmt: skip
    rng = np.random.default_rng(SEED)
    r0 = rng.uniform(size=(lanes, N_PART, DIM)) @ basis
    v0 = rng.normal(scale=0.03, size=(lanes, N_PART, DIM))
    keys = np.stack([make_key(i) for i in range(lanes)])
    # device-resident state (CUDA tensors) for the device number; NumPy in/out for e2e
    lane0 = init_state(energy, waves, basis, torch.from_numpy(r0).cuda(), torch.from_numpy(v0).cuda(),
                       np.full(lanes, 1e-3), keys, st)  # fmt: skip
    host0 = init_state(energy, waves, basis, r0, v0, np.full(lanes, 1e-3), keys, st)
    for _ in range(args.warmup):
        simulate(energy, waves, basis, st, lane0, max(n_steps // 10, 1))
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        res = simulate(energy, waves, basis, st, lane0, n_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    value = lanes * n_steps / (ms / 1e3)
    t0 = time.perf_counter()
    simulate(energy, waves, basis, st, host0, n_steps)
    e2e_s = time.perf_counter() - t0
    buf_bytes = sum(int(np.asarray(x).nbytes) for x in (host0.snap.r, host0.snap.rho, host0.snap.wind_abs,
                                                        host0.snap.wind_net, host0.trace.rho, host0.r,
                                                        host0.v, host0.f, host0.rho_prev))  # fmt: skip
    w = int(waves.n_vectors.shape[0])
    cpu_s = None if args.no_cpu_baseline else _md_host_sample(ks, basis, waves, r0[0], v0[0], 20)
    # device-side algorithmic flops per lane-step: force (F_PAIR N M) + fresh waves every 10 steps
    flops = lanes * n_steps * (F_PAIR[DIM] * N_PART * ks.n.shape[0] +
                               0.1 * 40.0 * N_PART * (w - waves.n_constrained))  # fmt: skip
    peak = fp64_peak_tflops()
    line = {
        "metric": "MD lane-steps/s (simulate: BAOAB + tracked-wave observables)", "value": value,
        "unit": "lane-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"md_segment_d{DIM}_n{N_PART}_chi{CHI}_lanes{lanes}_steps{n_steps}",
                   "waves": w, "constrained": int(waves.n_constrained), "wind_every": 10,
                   "snapshots": len(st.record_steps), "trace_rows": st.max_rho_records,
                   "final_status_running": int((res.state.status == 0).sum().item()),
                   "state": "device-resident (CUDA tensors)",
                   "wall_s_per_step": wall / args.steps},
        "roofline": {"kernel": "whole MD segment (evaluations + step + observables)", "bound": "fp64",
                     "achieved": flops / (ms / 1e3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                     "frac": flops / (ms / 1e3) / 1e12 / peak if peak else None,
                     "algorithmic": "F_PAIR N M per force + 40 flops per (fresh wave, particle) every 10 steps"},
        "e2e": {"value": lanes * n_steps / e2e_s, "unit": "lane-steps/s",
                "h2d_bytes_per_step": buf_bytes, "d2h_bytes_per_step": buf_bytes,
                "note": "simulate() with a NumPy state: one upload and one download of the state"},
        "cpu_baseline": None if cpu_s is None else {
            "value": 1.0 / cpu_s, "unit": "lane-steps/s", "cores": 1, "kind": "port",
            "sample": "oracle chain: 20 BAOAB steps of one lane, direct-sum forces and all waves' densities"},
        "clocks": clocks,
    }  # fmt: skip
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ analysis
def run_analysis(args) -> None:
    """S(k) (isotropic, the ground-state driver's 5 / 400 k-set) and the pair
    histogram + nearest neighbours of 256 configurations, d=2 N=1000."""
    import oracle
    import torch

    from xla_cco.analysis import isotropic_structure_factor, nearest_neighbor_distances, pair_distance_histogram
    from xla_cco.analysis.structure import _isotropic_kset

    torch.cuda.set_device(0)
    box, ks, energy = workload()
    basis = np.asarray(box.basis)
    b = args.batch
    s = np.random.default_rng(SEED).uniform(size=(b, N_PART, DIM))
    s_dev = torch.from_numpy(s).cuda()
    nv, _ = _isotropic_kset(basis, 5.0, 400.0)
    edges = np.linspace(0.0, 0.2 * np.sqrt(N_PART), 201)

    def one():
        isotropic_structure_factor(s_dev, box, 5.0, 400.0)
        pair_distance_histogram(s_dev, box, edges)
        for i in range(b):
            nearest_neighbor_distances(s_dev[i], box)

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    for _ in range(args.steps):
        isotropic_structure_factor(s_dev, box, 5.0, 400.0)
    e1.record(stream)
    for _ in range(args.steps):
        pair_distance_histogram(s_dev, box, edges)
    e2.record(stream)
    torch.cuda.synchronize()
    sk_ms = e0.elapsed_time(e1) / args.steps
    pr_ms = e1.elapsed_time(e2) / args.steps
    sk_pairs = b * N_PART * nv.shape[0]
    hist_pairs = b * N_PART * (N_PART - 1) / 2
    t0 = time.perf_counter()
    oracle.structure_factor_direct(s[0], nv[:2000])
    cpu_sk = (time.perf_counter() - t0) / (N_PART * 2000)
    t0 = time.perf_counter()
    oracle.min_image_distances(s[0], basis)
    cpu_pair = (time.perf_counter() - t0) / (N_PART * (N_PART - 1) / 2)
    line = {
        "metric": "isotropic S(k) (k, particle) pairs/s", "value": sk_pairs / (sk_ms / 1e3),
        "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sk_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"analysis_d{DIM}_n{N_PART}_b{b}", "sk_kvectors": int(nv.shape[0]),
                   "pair_histogram_ms": pr_ms, "pair_histogram_pairs_per_s": hist_pairs / (pr_ms / 1e3),
                   "g2_bins": 200},
        "cpu_baseline": {"value": 1.0 / cpu_sk, "unit": "pairs/s", "cores": 1, "kind": "port",
                         "sample": "oracle direct sum: 1 config x 2000 k; pair oracle 1 config",
                         "pair_histogram_pairs_per_s": 1.0 / cpu_pair},
    }  # fmt: skip
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ground-state driver
def run_cli(args) -> None:
    """The ground-state driver end to end (``python -m xla_cco.cli.relax``) on a
    ConfigPack of 256 seeded d=2 N=1000 configurations at chi = 0.40: read the
    pack, relax on the GPU, write the packs, S(k), g2, Hp tables and the log."""
    import tempfile

    import torch

    from xla_cco import ka_from_chi
    from xla_cco.cli import relax as cli
    from xla_cco.io import PackedConfig, write_configpack

    torch.cuda.set_device(0)
    b = args.batch
    rng = np.random.default_rng(SEED)
    names = (b"a\x00\x00\x00",) * N_PART
    cfgs = [PackedConfig(np.eye(DIM), rng.uniform(size=(N_PART, DIM)), 1.0, names) for _ in range(b)]
    with tempfile.TemporaryDirectory() as tmp:
        write_configpack(Path(tmp) / "in", cfgs)
        argv = ["--dim", str(DIM), "--ka", repr(ka_from_chi(CHI, PHI_PACK, DIM)), "--phi", str(PHI_PACK),
                "--load", str(Path(tmp) / "in"), "--save", str(Path(tmp) / "out"), "--batch-size", str(b)]
        for _ in range(args.warmup):
            cli.run(cli.build_parser().parse_args(argv))
        walls, logs = [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            logs.append(cli.run(cli.build_parser().parse_args(argv)))
            walls.append(time.perf_counter() - t0)
    wall = float(np.median(walls))
    log = logs[-1]
    line = {
        "metric": "ground-state driver: configurations/s end to end (read, relax, write, S(k), g2, Hp)",
        "value": b / wall, "unit": "configs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"cli_relax_d{DIM}_n{N_PART}_chi{CHI}_b{b}", "M": log["M"],
                   "n_success": log["n_success"], "stage_seconds": log["wall_seconds"],
                   "timing": "host wall clock around cli.run, median over steps"},
    }  # fmt: skip
    print(json.dumps(line), flush=True)


def kernel_timeline(call, n: int, d: int, batch: int) -> dict:
    """Kernel records (CUPTI, through torch.profiler) of one relaxation call:
    µs per launch per kernel, the span from the first kernel's start to the
    last one's end, and the time at least one kernel ran, per tick."""
    import re

    import torch
    from torch.profiler import ProfilerActivity, profile

    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        out = call()
        torch.cuda.synchronize()
    rec = sorted((e.time_range.start, e.time_range.end, e.name) for e in prof.events()
                 if e.device_type == torch.autograd.DeviceType.CUDA)  # fmt: skip
    per: dict = {}
    for t0, t1, name in rec:
        m = re.search(r"(k_\w+|Memcpy \w+)(<[^>]*>)?", name)
        key = m.group(0) if m else name[:40]
        c = per.setdefault(key, [0, 0.0])
        c[0] += 1
        c[1] += t1 - t0
    busy, cs, ce = 0.0, rec[0][0], rec[0][1]
    for t0, t1, _ in rec[1:]:
        if t0 > ce:
            busy += ce - cs
            cs, ce = t0, t1
        else:
            ce = max(ce, t1)
    busy += ce - cs
    ticks = max(int(out["ticks"]), 1)
    return {"profile": "timeline", "n": n, "d": d, "batch": batch, "ticks": ticks,
            "span_us_per_tick": (rec[-1][1] - rec[0][0]) / ticks, "busy_us_per_tick": busy / ticks,
            "us_per_launch": {k: round(v[1] / v[0], 2)
                              for k, v in sorted(per.items(), key=lambda kv: -kv[1][1])}}  # fmt: skip


def run_profile(args) -> None:
    """Kernel-level profiling driver (run under ncu).
    --profile-shape N,d,chi profiles another system than the headline one.
    Without ncu it prints the device time per evaluation (eval mode) or per
    relaxation and tick (relax mode, CUDA events; the first rep includes the
    schedule tuning)."""
    import torch

    from xla_cco import LBFGSSettings
    from xla_cco.minimize import relax_device
    from xla_cco.workloads import energy_for

    if args.profile_shape:
        n_s, d_s, chi_s = args.profile_shape.split(",")
        n, d = int(n_s), int(d_s)
        energy = energy_for(n, d, float(chi_s))
    else:
        n, d = N_PART, DIM
        _, _, energy = workload()
    s0 = np.random.default_rng(SEED).uniform(size=(args.batch, n, d))
    s_dev = torch.from_numpy(s0).cuda()
    if args.profile == "eval":
        energy.evaluate(s_dev)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.reps):
            energy.evaluate(s_dev)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.reps
        m = int(energy._rows.size)
        tf = args.batch * n * m * F_PAIR[d] / (ms * 1e-3) / 1e12
        print(json.dumps({"profile": "eval", "n": n, "d": d, "m": m, "batch": args.batch,
                          "ms_per_eval": ms, "tflops": tf}), flush=True)
    elif args.timeline:
        # CUPTI kernel records of one relaxation (after one untimed run):
        # per-kernel time per launch and the device's busy share of the span
        settings = LBFGSSettings(energy_tol=TOL, max_evals_per_pass=args.timeline_evals)
        relax_device(energy, s_dev, settings)
        torch.cuda.synchronize()
        print(json.dumps(kernel_timeline(lambda: relax_device(energy, s_dev, settings), n, d,
                                         args.batch)), flush=True)
    else:
        for _ in range(args.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            out = relax_device(energy, s_dev, LBFGSSettings(energy_tol=TOL))
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            ticks = int(out["ticks"])
            print(json.dumps({"profile": "relax", "n": n, "d": d, "batch": args.batch, "ms": ms,
                              "ticks": ticks, "us_per_tick": 1e3 * ms / max(ticks, 1),
                              "evals_per_lane": [int(v) for v in out["n_evals"].tolist()][:8],
                              "schedule": list(out["schedule"])}), flush=True)
    torch.cuda.synchronize()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cco", "reference"], default="cco")
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-target", action="store_true",
                    help="skip the mixed-ensemble comparison the default N=1 line carries")
    ap.add_argument("--profile", choices=["eval", "relax"], default=None,
                    help="profiling driver for ncu: run the kernels only")  # fmt: skip
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--profile-shape", default=None, help="N,d,chi of the profiled system")
    ap.add_argument("--timeline", action="store_true",
                    help="relax profiling: CUPTI kernel records of one relaxation (torch.profiler)")
    ap.add_argument("--timeline-evals", type=int, default=300,
                    help="max_evals_per_pass of the --timeline relaxation")
    ap.add_argument("--md-lanes", type=int, default=64)
    ap.add_argument("--md-steps", type=int, default=2000)
    ap.add_argument("--workload", choices=["batch", "descent", "mixed", "serve", "precision", "md", "analysis",
                                           "cli"],
                    default="batch",
                    help="batch: the headline 256-lane d2 N1000 relax; mixed: the 512-instance "
                         "mixed-size ensemble; serve: a Poisson request stream")  # fmt: skip
    ap.add_argument("--mixed-count", type=int, default=512)
    ap.add_argument("--plain-sample", type=int, default=0, help="0: every instance")
    ap.add_argument("--served", action="store_true",
                    help="mixed workload: also serve the ensemble with mixed precision")  # fmt: skip
    ap.add_argument("--serve-count", type=int, default=200)
    ap.add_argument("--precision-batch", type=int, default=64)
    ap.add_argument("--serve-precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-branches", type=int, default=0,
                    help="graph branches of the serving pool (0: its own choice by live lanes)")
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
    elif args.workload == "descent" and args.impl == "cco":
        run_descent(args)
    elif args.workload == "mixed" and args.impl == "cco":
        run_mixed(args)
    elif args.workload == "serve" and args.impl == "cco":
        run_serve(args)
    elif args.workload == "precision" and args.impl == "cco":
        run_precision(args)
    elif args.workload == "md" and args.impl == "cco":
        run_md(args)
    elif args.workload == "analysis" and args.impl == "cco":
        run_analysis(args)
    elif args.workload == "cli" and args.impl == "cco":
        run_cli(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_device(args)


if __name__ == "__main__":
    main()
