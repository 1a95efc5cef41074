#!/usr/bin/env python
"""Band-path benchmark: k-points/s of mixed-precision batched CISS.

Workload (default ``c2``): seeded synthetic 3D bundle, 1000 atoms x 13
orbitals (n = 13000, nnz = 15.7M), 121-point Y-G-X-M path, 32 contour
nodes, 32 probes, 4 moments, a window holding ~100 states at Gamma.  One
step = the whole Band hot path for ``--kpoints-per-step`` k points:
device Bloch sums, all shifted factorizations and solves (with FP64
refinement in mixed precision), moments, Rayleigh-Ritz and FP64 residuals.

Reported (one JSON line on rank 0):
  value        k-points/s of the chosen form, inputs resident on the GPU
  e2e          same through BandEngine with the operator block values copied
               from pinned host memory every step and energies read back
  plain        k-points/s of the plain complex64 one-node-per-factorization
               path with no refinement (the drop-in baseline)
  accuracy     max |E - E_FP64| over sampled k points (FP64 dense oracle)
  roofline     factorization (dominant, tensor/FP32 bound) achieved TFLOP/s
  cpu_baseline oracle CISS on the host cores for a bounded sample
``--impl reference`` times the reference algorithm on the host cores (the
oracle restatement; the reference's cuDSS extension does not install).
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
sys.path.insert(0, str(ROOT))

GUARD_EV = 0.02  # BandCalculation's continuity guard


def parse() -> argparse.Namespace:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--kpoints-per-step", type=int, default=0)
    ap.add_argument("--precision", choices=("mixed", "plain"), default="mixed")
    ap.add_argument("--tensor-cores", type=int, default=1)
    ap.add_argument("--plain-kpoints", type=int, default=1)
    ap.add_argument("--accuracy-kpoints", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--refinement-steps", type=int, default=-1,
                    help="FP64 refinement sweeps per mixed solve (-1 = engine default)")
    ap.add_argument("--max-pencils", type=int, default=0,
                    help="cap on pencils factored together (0 = by memory)")
    ap.add_argument("--ordering", choices=("auto", "natural", "nested_dissection"),
                    default="auto", help="tile-plan ordering when not autotuned")
    ap.add_argument("--autotune", type=int, default=1,
                    help="1: time candidate tile plans and k-point batches on the device first")
    ap.add_argument("--schur-depth", type=int, default=2, choices=(1, 2),
                    help="tile steps per tensor-core Schur pass (2 = K 256)")
    ap.add_argument("--lookahead-sms", type=int, default=0,
                    help="SMs left to the factorization's lookahead side stream (0 = default)")
    ap.add_argument("--solve-ctas", type=int, default=0, choices=(0, 1, 2),
                    help="CTAs per SM of the tensor-core solve update (0 = default)")
    ap.add_argument("--tensor-core-solves", type=int, default=-1,
                    help="1/0: split-BF16 tensor-core solve updates on/off (-1 = engine default)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int) -> None:
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        mhz, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(mhz)}


def workload(name: str):
    from aospectrum_b200 import synth
    from aospectrum_b200.kpath import kpath_from_dict

    w = synth.WORKLOADS[name]
    return w, kpath_from_dict(w.kpath)


def cpu_baseline(bundle, kpts, lo, hi, w, seconds_cap: float = 30.0) -> dict:
    """Oracle CISS on the host cores: reference Bloch restatement for one k
    plus one complex64 dense-LU shifted solve (LAPACK, all host threads);
    k-points/s extrapolated to the N solves a k point needs."""
    from oracle import bloch_ref, ciss_ref
    from scipy import sparse

    cores = len(os.sched_getaffinity(0))
    t0 = time.perf_counter()
    pat = bloch_ref.build_pattern(bundle)
    t_pattern = time.perf_counter() - t0
    t0 = time.perf_counter()
    h, s = bloch_ref.bloch_pair(pat, bundle, kpts[0])
    t_bloch = time.perf_counter() - t0
    n = bundle.n_orbitals
    hm = sparse.csr_matrix((h, pat.indices, pat.indptr), shape=(n, n))
    sm = sparse.csr_matrix((s, pat.indices, pat.indptr), shape=(n, n))
    shifts, nodes, weights = ciss_ref.contour(lo, hi, w.integration_points)
    q = ciss_ref.probes(n, w.block_size)
    rhs = np.asarray(sm @ q, dtype=np.complex64)
    t0 = time.perf_counter()
    ciss_ref.shifted_solve(hm, sm, shifts[0], rhs, method="dense")
    t_solve = time.perf_counter() - t0
    per_k = t_bloch + w.integration_points * t_solve
    return {"value": 1.0 / per_k, "unit": "k-points/s", "cores": cores, "kind": "port",
            "sample": (f"oracle Bloch sum of 1 k point ({t_bloch:.2f} s) + 1 of "
                       f"{w.integration_points} complex64 dense-LU shifted solves "
                       f"({t_solve:.2f} s, n={n}, {w.block_size} rhs); k-points/s = "
                       f"1/(t_bloch + {w.integration_points} t_solve); pattern build "
                       f"{t_pattern:.2f} s once")}


METRIC = "k-points/s at <=1e-4 eV vs FP64 (mixed+batched CISS, 1 B200)"


def reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w, kp = workload(args.workload)
    from aospectrum_b200 import synth

    bundle = synth.generate_bundle(w.spec)
    lo, hi = w.window_ev[0] - GUARD_EV, w.window_ev[1] + GUARD_EV
    kpts = kp.fractional_points
    times = []
    base = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        base = cpu_baseline(bundle, [kpts[i % len(kpts)]], lo, hi, w)
        if i >= args.warmup:
            times.append(1.0 / base["value"])
    per_k = float(np.mean(times))
    value = 1.0 / per_k
    # same metric, unit and config as this file's own arm; "impl" and
    # cpu_baseline say that the host reference algorithm produced the value
    out = {"metric": METRIC, "value": value,
           "unit": "k-points/s", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": per_k * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
           "config": {"workload": f"{w.name}: {w.notes}", "n": w.spec.n_orbitals,
                      "integration_points": w.integration_points, "block_size": w.block_size,
                      "moment_size": w.moment_size},
           "cpu_baseline": {**base, "value": value},
           "e2e": {"value": value, "unit": "k-points/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def serving_arm(args) -> None:
    """Serving stream (c4, reduced sizes): seeded Poisson arrivals of band
    requests over 216-1000-atom bundles through BandServer (continuous
    batching, mixed precision), against serial plain solves of the same
    requests on the same GPU."""
    import torch

    from aospectrum_b200 import synth
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine
    from aospectrum_b200.kpath import kpath_from_dict
    from aospectrum_b200.serve import BandRequest, BandServer, percentile

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = synth.serving_stream()
    kpts = kpath_from_dict(synth.YGXM).fractional_points
    settings = CissSettings()
    bundles, windows = {}, {}
    for r in stream:
        key = r.spec.name
        if key not in bundles:
            bundles[key] = synth.generate_bundle(r.spec)
        wk = (key, r.states)
        if wk not in windows:
            h, s = synth.dense_gamma(bundles[key])
            hd = torch.from_numpy(h).to(dev)
            sd = torch.from_numpy(s).to(dev)
            lc = torch.linalg.cholesky(sd)
            li = torch.linalg.solve_triangular(lc, torch.eye(h.shape[0], dtype=hd.dtype,
                                                             device=dev), upper=False)
            e = np.sort(torch.linalg.eigvalsh(li @ hd @ li.T).cpu().numpy())
            c = float(np.median(e))
            dist = np.sort(np.abs(e - c))
            half = 0.5 * (dist[r.states - 1] + dist[r.states])
            windows[wk] = (c - half, c + half)
            del hd, sd, lc, li
            torch.cuda.empty_cache()
    reqs = [BandRequest(bundles[r.spec.name], [kpts[i] for i in r.kpoint_indices],
                        EnergyInterval(*windows[(r.spec.name, r.states)]), settings,
                        f"r{i}") for i, r in enumerate(stream)]
    total_k = sum(len(r.kpoint_indices) for r in stream)
    # continuous batching: submit at the seeded arrival times
    with BandServer(device=dev, slots=4, engine_settings=EngineSettings(precision="mixed")) as srv:
        t0 = time.perf_counter()
        futs = []
        for r, q in zip(stream, reqs):
            delay = r.arrival_s - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            futs.append(srv.submit(q))
        responses = [f.result() for f in futs]
        span = time.perf_counter() - t0
        stats = srv.stats()
    # serial plain baseline: one request at a time, plain complex64 batched
    # engine, arrivals replayed on the same clock
    serial_lat = []
    engines = {}
    t0 = time.perf_counter()
    for r, q in zip(stream, reqs):
        now = time.perf_counter() - t0
        if now < r.arrival_s:
            time.sleep(r.arrival_s - now)
        key = r.spec.name
        if key not in engines:
            engines[key] = BandEngine(q.bundle, settings, EngineSettings(precision="plain"),
                                      device=dev)
        engines[key].solve_kpoints(q.kpoints, q.interval)
        torch.cuda.synchronize(dev)
        serial_lat.append(time.perf_counter() - t0 - r.arrival_s)
    serial_span = time.perf_counter() - t0
    for e in engines.values():
        e.close()
    lat = [x.latency_seconds for x in responses]
    out = {"metric": "serving k-points/s with p50/p99 latency (continuous batching, 1 B200)",
           "value": total_k / span, "unit": "k-points/s", "n_gpus": 1, "steps": 1, "warmup": 0,
           "ms_per_step": span * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c64+bf16x3 tensor-core updates, fp64 refinement",
           "data": "synthetic (seeded serving stream)",
           "config": {"workload": "c4 serving stream, reduced sizes: 12 requests, 216-1000-atom "
                                  "cubic bundles, 5 or 13 orbitals, 4-16 k points, windows of "
                                  "20-60 Gamma states, Poisson arrivals at 2/s",
                      "requests": len(stream), "kpoints": total_k, "slots": 4,
                      "bundles": sorted({r.spec.name for r in stream})},
           "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
           "server_stats": stats,
           "serial_plain": {"kpoints_per_s": total_k / serial_span,
                            "p50_latency_s": percentile(serial_lat, 50),
                            "p99_latency_s": percentile(serial_lat, 99)},
           "max_residual_ev": max(x.maximum_residual_ev for x in responses)}
    print(json.dumps(out), flush=True)


def main() -> None:
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.workload == "c4":
        serving_arm(args)
        return
    import torch
    import torch.distributed as dist

    from aospectrum_b200 import native, synth
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=dev)
    if args.lookahead_sms:
        native.library().aosb_factor_set_lookahead_sms(args.lookahead_sms)
    if args.solve_ctas:
        native.library().aosb_solve_set_ctas_per_sm(args.solve_ctas)
    w, kp = workload(args.workload)
    bundle = synth.generate_bundle(w.spec)
    interval = EnergyInterval(w.window_ev[0] - GUARD_EV, w.window_ev[1] + GUARD_EV)
    settings = CissSettings(integration_points=w.integration_points, block_size=w.block_size,
                            moment_size=w.moment_size)
    eng = BandEngine(bundle, settings,
                     EngineSettings(precision=args.precision,
                                    tensor_cores=bool(args.tensor_cores),
                                    autotune=bool(args.autotune),
                                    ordering=args.ordering,
                                    schur_depth=args.schur_depth,
                                    max_pencils=args.max_pencils,
                                    **({"refinement_steps": args.refinement_steps}
                                       if args.refinement_steps >= 0 else {}),
                                    **({"tensor_core_solves": bool(args.tensor_core_solves)}
                                       if args.tensor_core_solves >= 0 else {})), device=dev)
    kpts = kp.fractional_points
    tuning = eng.tuning.as_dict() if eng.tuning is not None else None
    if args.kpoints_per_step:
        nk_step = args.kpoints_per_step
    elif args.autotune:
        from aospectrum_b200.autotune import tune_batch

        mine = kpts[rank::world]
        nk_step, rates = tune_batch(eng, mine[:4], interval,
                                    sizes=(1, 2, 4) if w.spec.n_orbitals > 4000 else (4, 8, 16))
        tuning = dict(tuning or {}, kpoints_per_batch=nk_step,
                      kpoints_per_s_by_batch={str(k): round(v, 4) for k, v in rates.items()})
    else:
        nk_step = 1 if w.spec.n_orbitals > 4000 else 8
    if world > 1:
        # every rank runs the same batch (the smallest any rank chose), so
        # the work count below holds for all of them
        t = torch.tensor([nk_step], dtype=torch.int64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        nk_step = int(t.item())

    def kset(step: int) -> np.ndarray:
        # weak scaling: rank r owns k indices r, r+N, ...; each step takes nk_step of them
        mine = kpts[rank::world]
        idx = [(step * nk_step + j) % len(mine) for j in range(nk_step)]
        return mine[idx]

    def barrier():
        if world > 1:
            dist.barrier()

    for i in range(args.warmup):
        eng.solve_kpoints(kset(i), interval)
    torch.cuda.synchronize(dev)
    launches0 = native.library().aosb_launch_count()
    eng.profile_factor = True
    eng.factor_times_ms = []
    native.library().aosb_kernel_timing(1)
    barrier()
    torch.cuda.synchronize(dev)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record()
        results = []
        for i in range(args.steps):
            res, _ = eng.solve_kpoints(kset(args.warmup + i), interval)
            results.append(res)
        stop.record()
        torch.cuda.synchronize(dev)
    barrier()
    elapsed = start.elapsed_time(stop) / 1e3
    launches = native.library().aosb_launch_count() - launches0
    eng.profile_factor = False
    k_ms, k_flops, k_bytes, k_launches = (native.C.c_double(), native.C.c_double(),
                                          native.C.c_double(), native.c_i64())
    native.library().aosb_kernel_timing_read(native.C.byref(k_ms), native.C.byref(k_flops),
                                             native.C.byref(k_bytes), native.C.byref(k_launches))
    breakdown = {}
    peaks_hbm = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()).get("hbm_gbs", 6650.0) \
        if (ROOT / "MEASURED_PEAKS.json").exists() else 6650.0
    for cat, name in ((1, "solve_diag"), (2, "solve_update"), (3, "fp64_residual"),
                      (4, "fp64_spmm"), (5, "bloch_sum")):
        c_ms, c_fl, c_by, c_n = (native.C.c_double(), native.C.c_double(), native.C.c_double(),
                                 native.c_i64())
        native.library().aosb_kernel_timing_read_category(
            cat, native.C.byref(c_ms), native.C.byref(c_fl), native.C.byref(c_by),
            native.C.byref(c_n))
        if c_n.value:
            breakdown[name] = {"ms_per_step": c_ms.value / args.steps, "launches": int(c_n.value),
                               "avg_launch_us": 1e3 * c_ms.value / c_n.value,
                               "gbs": c_by.value / (c_ms.value / 1e3) / 1e9,
                               "hbm_frac": (c_by.value / (c_ms.value / 1e3) / 1e9) /
                               peaks_hbm,
                               "tflops": c_fl.value / (c_ms.value / 1e3) / 1e12}
    breakdown["schur_tc"] = {"ms_per_step": k_ms.value / args.steps,
                             "launches": int(k_launches.value)}
    native.library().aosb_kernel_timing(0)
    t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    elapsed = float(t.item())
    total_k = world * args.steps * nk_step
    value = total_k / elapsed
    stats = dict(eng.last_stats)
    info = eng.plan.info
    # roofline of the dominant kernel: the tensor-core Schur update
    # (schur_tc_kernel), timed with CUDA events on its launch stream over the
    # timed region; algorithmic flops = 8 T^3 per (target tile, pencil).
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (
        ROOT / "MEASURED_PEAKS.json").exists() else {}
    tc = args.precision == "mixed" and bool(args.tensor_cores)
    ft = eng.factor_times_ms
    factor_tflops = (info.factor_flops_alg * float(np.mean(eng.factor_pencils)) /
                     (float(np.mean(ft)) / 1e3) / 1e12) if ft else None
    if tc and k_launches.value > 0:
        sustained = peaks.get("bf16_tflops_sustained")
        peak = (sustained if sustained else 1400.0) / 3.0
        achieved = k_flops.value / (k_ms.value / 1e3) / 1e12
        per_launch_targets = k_flops.value / k_launches.value / (8.0 * info.tile ** 3)
        traffic = schur_traffic_per_target()
        roofline = {
            "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak,
            "traffic": traffic * per_launch_targets if traffic else None,
            "kernel": "schur_tc_kernel",
            "launches": int(k_launches.value),
            "avg_launch_ms": k_ms.value / k_launches.value,
            "algorithmic_flops_per_launch": k_flops.value / k_launches.value,
            "algorithmic_bytes_per_launch": k_bytes.value / k_launches.value,
            "achieved_hbm_gbs": k_bytes.value / (k_ms.value / 1e3) / 1e9,
            "hbm_peak_gbs": peaks.get("hbm_gbs", 6650.0),
            "peak_source": ("of measured: MEASURED_PEAKS.json bf16_tflops_sustained / 3 "
                            "(split BF16 issues 3 products per algorithmic product)"
                            if sustained else "of fallback: 1400 TFLOP/s sustained / 3"),
            "factorization_tflops": factor_tflops,
            "flops_per_factorization": info.factor_flops_alg}
    else:
        peak = 74.4
        roofline = {"bound": "fp32-simt", "achieved": factor_tflops, "peak": peak,
                    "unit": "TFLOP/s", "frac": (factor_tflops / peak) if factor_tflops else None,
                    "traffic": None, "kernel": "tile LU factorization (FP32 SIMT)",
                    "peak_source": "nominal FP32 SIMT 148 SM x 128 lanes x 2 x 1.965 GHz",
                    "flops_per_factorization": info.factor_flops_alg}
    out = {
        "metric": METRIC,
        "value": value, "unit": "k-points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": ("c64+bf16x3 tensor-core updates, fp64 refinement" if tc else
                  ("c64 fp32 updates, fp64 refinement" if args.precision == "mixed" else "c64")),
        "data": "synthetic (seeded generator)",
        "config": {"workload": f"{w.name}: {w.notes}", "n": w.spec.n_orbitals, "nnz": info.nnz,
                   "kpoints_per_step": nk_step, "integration_points": w.integration_points,
                   "block_size": w.block_size, "moment_size": w.moment_size,
                   "window_ev": list(w.window_ev), "precision": args.precision,
                   "tile": info.tile, "ordering": eng.plan.ordering,
                   "refinement_steps": eng.engine.refinement_steps if args.precision == "mixed"
                   else 0,
                   "tensor_core_solves": bool(eng.engine.tensor_core_solves),
                   "schur_depth": eng.engine.schur_depth,
                   "lookahead_sms": args.lookahead_sms or "default",
                   "solve_ctas_per_sm": args.solve_ctas or "default",
                   "autotune": tuning,
                   "factorizations_per_step": stats.get("factorizations"),
                   "pencil_batch": stats.get("pencil_batch"),
                   "l2": "inputs larger than L2 (factor storage %.2f GB per pencil)" % (
                       info.factor_bytes / 1e9),
                   "parallelism": f"dp{world} (k points sharded)"},
        "gpu_launches": int(launches),
        "kernel_event_times": breakdown,
        "clocks": clocks.summary(),
        "roofline": roofline,
    }
    total_mem = torch.cuda.get_device_properties(dev).total_memory
    out["memory"] = {"peak_allocated_gb": torch.cuda.max_memory_allocated(dev) / 1e9,
                     "factor_gb_per_pencil": info.factor_bytes / 1e9,
                     "factor_gb_resident": info.factor_bytes * stats.get("pencil_batch", 1) / 1e9,
                     "device_total_gb": total_mem / 1e9}
    if rank == 0:
        out["stage_seconds_last_step"] = {k: round(v, 4) for k, v in
                                          stats.get("stage_seconds", {}).items()}
        out["per_k_stage_seconds"] = {k: round(v, 4) for k, v in
                                      results[-1][0].stage_seconds.items()}
        # accuracy vs FP64 dense generalized eigenvalues (sampled k points);
        # above n = 20000 a dense FP64 eigensolve does not fit, and the check
        # is the device FP64 eigenpair residuals plus agreement with the
        # plain complex64 path at the same k (below)
        errs = []
        dense_ok = w.spec.n_orbitals <= 20000
        for i in range(min(args.accuracy_kpoints, len(kpts)) if dense_ok else 0):
            kpt = kpts[(i * 37) % len(kpts)]
            res, _ = eng.solve_kpoints([kpt], interval)
            pair = eng.host_pair(kpt)
            exact = fp64_window(pair, interval, dev)
            got = np.sort(res[0].energies_ev.astype(np.float64))
            if got.size != exact.size:
                errs.append(float("inf"))
            else:
                errs.append(float(np.max(np.abs(got - exact))) if got.size else 0.0)
        out["accuracy"] = {"max_eig_error_ev": max(errs) if errs else None,
                           "kpoints_checked": len(errs),
                           "max_residual_ev": max(r.maximum_residual_ev for rs in results
                                                  for r in rs),
                           "oracle": ("FP64 dense generalized eigh (torch, cuSOLVER) of the "
                                      "same H(k), S(k)" if dense_ok else
                                      "FP64 eigenpair residuals on the device; dense FP64 "
                                      "eigh does not fit at this n")}
        # plain complex64 per-shift baseline on the same GPU: one shift per
        # factorization call, no refinement (the reference's
        # contour_batch_size = 1 form); the batched plain path for context
        if args.plain_kpoints > 0 and args.precision == "mixed":
            plain_energies = {}
            plain_residuals = []

            def plain_rate(max_pencils: int, warm: bool = True) -> float:
                plain = BandEngine(bundle, settings,
                                   EngineSettings(precision="plain", max_pencils=max_pencils),
                                   device=dev)
                if warm:
                    plain.solve_kpoints(kset(0)[:1], interval)
                torch.cuda.synchronize(dev)
                t0 = time.perf_counter()
                for i in range(args.plain_kpoints):
                    res, _ = plain.solve_kpoints(kset(1 + i)[:1], interval)
                    plain_energies[i] = np.sort(res[0].energies_ev.astype(np.float64))
                    plain_residuals.append(res[0].maximum_residual_ev)
                torch.cuda.synchronize(dev)
                tp = (time.perf_counter() - t0) / args.plain_kpoints
                plain.close()
                return 1.0 / tp

            large = w.spec.n_orbitals > 20000
            per_shift = plain_rate(1, warm=not large)
            batched = plain_rate(0, warm=not large) if not large else None
            out["plain"] = {"value": per_shift, "unit": "k-points/s",
                            "max_residual_ev": max(plain_residuals) if plain_residuals else None,
                            "note": "complex64, one shift per factorization call, no refinement",
                            "batched_value": batched,
                            "batched_note": "complex64, all shifts of a k point in one batched "
                                            "call, no refinement"}
            out["speedup_vs_plain"] = value / world / per_shift
            if batched:
                out["speedup_vs_plain_batched"] = value / world / batched
            # mixed vs plain complex64 eigenvalues at the same k points
            diffs = []
            for i, ep in plain_energies.items():
                res, _ = eng.solve_kpoints(kset(1 + i)[:1], interval)
                em = np.sort(res[0].energies_ev.astype(np.float64))
                diffs.append(float(np.max(np.abs(em - ep))) if em.size == ep.size and em.size
                             else (0.0 if em.size == ep.size else float("inf")))
            out["accuracy"]["max_diff_vs_plain_c64_ev"] = max(diffs) if diffs else None
        # end to end through the public engine API with host buffers
        if not args.no_e2e:
            out["e2e"] = e2e_leg(eng, bundle, kset, interval, args)
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(bundle, [kpts[0]], interval.lower_ev,
                                               interval.upper_ev, w)
        print(json.dumps(out), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


def schur_traffic_per_target() -> float | None:
    """DRAM bytes per (target tile, pencil) of schur_tc_kernel from the
    committed ncu capture summary (dram__bytes_read.sum + write.sum of one
    launch divided by the targets it updated)."""
    f = ROOT / "profiles" / "schur_tc_kernel_c2.json"
    if not f.exists():
        return None
    return float(json.loads(f.read_text())["dram_bytes_per_target"])


def fp64_window(pair, interval, dev) -> np.ndarray:
    import torch

    n = pair.n_orbitals
    hd = torch.from_numpy(pair.hamiltonian.toarray().astype(np.complex128)).to(dev)
    sd = torch.from_numpy(pair.overlap.toarray().astype(np.complex128)).to(dev)
    hd = 0.5 * (hd + hd.conj().T)
    sd = 0.5 * (sd + sd.conj().T)
    lc = torch.linalg.cholesky(sd)
    linv = torch.linalg.solve_triangular(lc, torch.eye(n, dtype=hd.dtype, device=dev),
                                         upper=False)
    e = torch.linalg.eigvalsh(linv @ hd @ linv.conj().T).cpu().numpy()
    del hd, sd, lc, linv
    torch.cuda.empty_cache()
    return np.sort(e[(e > interval.lower_ev) & (e < interval.upper_ev)])


def e2e_leg(eng, bundle, kset, interval, args) -> dict:
    """Public-API path with host buffers: every step copies the bundle's
    block values from pinned host memory into the engine and reads the
    energies back."""
    import torch

    hv = torch.from_numpy(np.array(bundle.operators.h_values)).pin_memory()
    sv = torch.from_numpy(np.array(bundle.operators.s_values)).pin_memory()
    steps = max(1, args.steps)
    eng.load_values(hv, sv)
    eng.solve_kpoints(kset(0), interval)
    torch.cuda.synchronize()
    d2h = 0
    t0 = time.perf_counter()
    for i in range(steps):
        eng.load_values(hv, sv)
        res, _ = eng.solve_kpoints(kset(i), interval)
        d2h += sum(r.energies_ev.nbytes for r in res)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    nk = len(kset(0))
    return {"value": nk / dt, "unit": "k-points/s",
            "h2d_bytes_per_step": int(hv.numel() * hv.element_size() + sv.numel() *
                                      sv.element_size()),
            "d2h_bytes_per_step": int(d2h / steps),
            "path": "BandEngine.load_values (pinned host) + solve_kpoints"}


if __name__ == "__main__":
    main()
