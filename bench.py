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
    ap.add_argument("--no-fp64-sample", action="store_true",
                    help="reference arm: skip the complex128 SuperLU shift-invert sample")
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
    ap.add_argument("--schur-pairs", type=int, default=-1, choices=(-1, 0, 1),
                    help="two-CTA (M = 256) pair Schur updates: 1 on, 0 off, -1 library default")
    ap.add_argument("--cuda-graphs", type=int, default=-1, choices=(-1, 0, 1),
                    help="replay each batch's triangular sweeps from a CUDA graph: 1 on, 0 off, "
                         "-1 engine default")
    ap.add_argument("--solve-lookahead", type=int, default=-1, choices=(-1, 0, 1),
                    help="next diagonal solve on a side stream: 1 on, 0 off, -1 library default")
    ap.add_argument("--solve-ctas", type=int, default=0, choices=(0, 1, 2),
                    help="CTAs per SM of the tensor-core solve update (0 = default)")
    ap.add_argument("--tensor-core-solves", type=int, default=-1,
                    help="1/0: split-BF16 tensor-core solve updates on/off (-1 = engine default)")
    ap.add_argument("--stream", choices=("reduced", "full"), default="reduced",
                    help="c4 serving stream sizes")
    ap.add_argument("--requests", type=int, default=0,
                    help="c4: requests of the seeded stream (0: 12 reduced, 6 full)")
    ap.add_argument("--fp64-check", type=int, default=2,
                    help="k points refined in FP64 (fp64check) when dense FP64 eigh does not fit")
    ap.add_argument("--fp64-check-interval", choices=("solve", "window"), default="solve",
                    help="interval of the FP64 check: the solve interval (window plus the "
                         "0.02 eV continuity guards) or the window alone")
    ap.add_argument("--accuracy-sweep", default="",
                    help="k indices ('all', 'a:b:s' or 'i,j,...'): no timing; per k point, "
                         "mixed and plain eigenvalues and residuals against FP64 dense eigh")
    ap.add_argument("--sweep-out", default="",
                    help="file for the per-k accuracy record (JSON); default stdout only")
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


class HostPath:
    """The oracle's CPU restatement of the Band path for one workload, on
    the host cores, split into the units that are timed: the pattern build
    (once per bundle), the Bloch sum of one k point, one complex64 dense-LU
    shifted solve (LAPACK on all host threads; a k point needs N of them),
    the CISS subspace phase (compression, Rayleigh-Ritz, ghost filter,
    residuals) of one k point, and optionally one complex128 SuperLU
    factorization + solve of a shifted pencil (the scipy FP64 shift-invert
    oracle)."""

    def __init__(self, bundle, w, lo: float, hi: float, kpt) -> None:
        from oracle import bloch_ref, ciss_ref
        from scipy import sparse

        self.w, self.lo, self.hi = w, lo, hi
        self.cores = len(os.sched_getaffinity(0))
        t0 = time.perf_counter()
        pat = bloch_ref.build_pattern(bundle)
        self.t_pattern = time.perf_counter() - t0
        t0 = time.perf_counter()
        h, s = bloch_ref.bloch_pair(pat, bundle, kpt)
        self.t_bloch = time.perf_counter() - t0
        n = self.n = bundle.n_orbitals
        self.h = sparse.csr_matrix((h, pat.indices, pat.indptr), shape=(n, n))
        self.s = sparse.csr_matrix((s, pat.indices, pat.indptr), shape=(n, n))
        self.shifts, self.nodes, self.weights = ciss_ref.contour(lo, hi, w.integration_points)
        self.rhs = np.asarray(self.s @ ciss_ref.probes(n, w.block_size), dtype=np.complex64)
        self.mom = np.zeros((n, w.block_size * w.moment_size), dtype=np.complex64)
        self.solve_times: list[float] = []
        self.t_subspace = None
        self.t_splu = None

    def solve(self, j: int) -> float:
        """One shifted solve (node j), accumulated into the moments."""
        from oracle import ciss_ref

        j %= self.w.integration_points
        t0 = time.perf_counter()
        x = ciss_ref.shifted_solve(self.h, self.s, self.shifts[j], self.rhs, method="dense")
        ciss_ref.accumulate_moments(self.mom, x, self.weights[j], self.nodes[j],
                                    self.w.block_size, self.w.moment_size)
        dt = time.perf_counter() - t0
        self.solve_times.append(dt)
        return dt

    def subspace(self) -> float:
        """The subspace phase on the moments accumulated so far (the same
        arithmetic and sizes as with all N solves)."""
        from oracle import ciss_ref

        t0 = time.perf_counter()
        ciss_ref.subspace(self.h, self.s, self.mom, self.lo, self.hi, block=self.w.block_size,
                          moments=self.w.moment_size)
        self.t_subspace = time.perf_counter() - t0
        return self.t_subspace

    def splu_sample(self) -> float:
        from oracle import ciss_ref

        t0 = time.perf_counter()
        ciss_ref.shifted_solve(self.h, self.s, self.shifts[0], self.rhs, method="splu")
        self.t_splu = time.perf_counter() - t0
        return self.t_splu

    def per_k(self) -> float:
        """Seconds per k point: Bloch sum + N shifted solves (the measured
        mean) + subspace phase."""
        return (self.t_bloch + self.w.integration_points * float(np.mean(self.solve_times))
                + (self.t_subspace or 0.0))

    def describe(self) -> dict:
        n_pts = self.w.integration_points
        out = {"cores": self.cores,
               "measured": {"pattern_build_s": round(self.t_pattern, 3),
                            "bloch_sum_1k_s": round(self.t_bloch, 3),
                            "dense_c64_shifted_solves": len(self.solve_times),
                            "dense_c64_solve_mean_s": round(float(np.mean(self.solve_times)), 3),
                            "subspace_phase_s": (round(self.t_subspace, 3)
                                                 if self.t_subspace is not None else None)},
               "extrapolated": (f"k-points/s = 1/(bloch + {n_pts} x mean dense solve + "
                                f"subspace): the {n_pts} solves a k point needs are taken at "
                                f"the measured mean of {len(self.solve_times)}")}
        if self.t_splu is not None:
            out["measured"]["fp64_splu_shift_invert_s"] = round(self.t_splu, 2)
            out["fp64_shift_invert_kpoints_per_s"] = 1.0 / (
                self.t_bloch + n_pts * self.t_splu + (self.t_subspace or 0.0))
        return out


def cpu_baseline(bundle, kpts, lo, hi, w, solves: int = 2) -> dict:
    """The oracle on the host cores for a bounded sample of the workload:
    Bloch sum of one k point, ``solves`` complex64 dense-LU shifted solves
    and the subspace phase, extrapolated to the N solves of a k point."""
    host = HostPath(bundle, w, lo, hi, kpts[0])
    for j in range(solves):
        host.solve(j)
    host.subspace()
    d = host.describe()
    return {"value": 1.0 / host.per_k(), "unit": "k-points/s", "cores": d["cores"],
            "kind": "port",
            "sample": (f"oracle Band path on the host: Bloch sum of 1 k point, {solves} of "
                       f"{w.integration_points} complex64 dense-LU shifted solves (n={host.n}, "
                       f"{w.block_size} rhs), subspace phase; {d['extrapolated']}"),
            "measured": d["measured"]}


METRIC = "k-points/s at <=1e-4 eV vs FP64 (mixed+batched CISS, 1 B200)"


def reference_arm(args) -> None:
    """The reference algorithm on the host cores (the oracle restatement:
    the reference's cuDSS extension cannot be installed).  Setup (untimed
    by the step clock, measured and reported): pattern build, Bloch sum of
    one k point, and one complex128 SuperLU shift-invert sample.  Each step
    is one complex64 dense-LU shifted solve of the next contour node, so
    ms_per_step is the measured time of one step; after the steps the
    subspace phase is timed once.  ``value`` is the per-k-point rate these
    measured units give (Bloch + N solves at the measured mean + subspace),
    the same metric as this file's own arm."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w, kp = workload(args.workload)
    from aospectrum_b200 import synth

    bundle = synth.generate_bundle(w.spec)
    lo, hi = w.window_ev[0] - GUARD_EV, w.window_ev[1] + GUARD_EV
    kpts = kp.fractional_points
    host = HostPath(bundle, w, lo, hi, kpts[0])
    if not args.no_fp64_sample:
        host.splu_sample()
    for i in range(args.warmup):
        host.solve(i)
    host.solve_times.clear()
    for i in range(args.steps):
        host.solve(args.warmup + i)
    step_ms = float(np.mean(host.solve_times)) * 1e3
    host.subspace()
    value = 1.0 / host.per_k()
    d = host.describe()
    # same metric, unit and config as this file's own arm; "impl" and
    # cpu_baseline say that the host reference algorithm produced the value
    out = {"metric": METRIC, "value": value,
           "unit": "k-points/s", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
           "config": {"workload": f"{w.name}: {w.notes}", "n": w.spec.n_orbitals,
                      "integration_points": w.integration_points, "block_size": w.block_size,
                      "moment_size": w.moment_size},
           "step": ("one complex64 dense-LU shifted solve (LAPACK, all host threads) of one "
                    "contour node; value = 1 / (bloch + N x mean step + subspace)"),
           "cpu_baseline": {"value": value, "unit": "k-points/s", "cores": d["cores"],
                            "kind": "port",
                            "sample": (f"{args.steps} timed shifted solves after "
                                       f"{args.warmup} warm-up; {d['extrapolated']}"),
                            "measured": d["measured"]},
           "e2e": {"value": value, "unit": "k-points/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    if "fp64_shift_invert_kpoints_per_s" in d:
        out["fp64_shift_invert"] = {
            "value": d["fp64_shift_invert_kpoints_per_s"], "unit": "k-points/s",
            "sample": "one complex128 SuperLU factorization + solve of a shifted pencil "
                      "(scipy, single-threaded), extrapolated to N per k point"}
    print(json.dumps(out), flush=True)


def serving_window(bundle, states: int, dev) -> tuple[float, float]:
    """Window around the median Gamma eigenvalue holding ``states`` states.
    Up to n = 16000 from the FP64 dense Gamma spectrum on the device; above,
    scaled from the dense spectrum of the 8x8x8 bundle with the same
    orbitals and generator (same on-site and hopping statistics): the
    density of states per orbital around its median, times n."""
    import torch

    from aospectrum_b200 import synth

    def spectrum(b):
        h, s = synth.dense_gamma(b)
        hd = torch.from_numpy(h).to(dev)
        sd = torch.from_numpy(s).to(dev)
        lc = torch.linalg.cholesky(sd)
        li = torch.linalg.solve_triangular(lc, torch.eye(h.shape[0], dtype=hd.dtype, device=dev),
                                           upper=False)
        e = np.sort(torch.linalg.eigvalsh(li @ hd @ li.T).cpu().numpy())
        del hd, sd, lc, li
        torch.cuda.empty_cache()
        return e

    n = bundle.n_orbitals
    if n <= 16000:
        e = spectrum(bundle)
        c = float(np.median(e))
        dist = np.sort(np.abs(e - c))
        half = 0.5 * (dist[states - 1] + dist[states])
        return c - half, c + half
    spec = bundle.provenance["spec"]
    small = synth.generate_bundle(synth.SyntheticSpec(**{
        **{k: tuple(v) if isinstance(v, list) else v for k, v in spec.items()},
        "name": spec["name"] + "-dos", "grid": (8, 8, 8), "cell": (19.2, 19.2, 19.2)}))
    e = spectrum(small)
    c = float(np.median(e))
    dist = np.sort(np.abs(e - c))
    probe = max(20, states * small.n_orbitals // n)
    width = float(dist[probe])           # half width holding `probe` states of the small bundle
    per_orbital = probe / (2.0 * width * small.n_orbitals)
    half = states / (2.0 * per_orbital * n)
    return c - half, c + half


def serving_arm(args) -> None:
    """Serving stream (c4): seeded Poisson arrivals of band requests through
    BandServer (continuous batching, mixed precision) against serial plain
    solves of the same requests on the same GPU.  ``--stream reduced``:
    216-1000-atom bundles, 4-16 k points, 20-60 states, 12 requests;
    ``--stream full``: the sizes the workload is specified with (216-8000
    atoms, 16-256 k points, 20-200 states; ``--requests`` of the seeded
    stream, 6 by default).  The serial plain baseline is measured: with
    ``full`` each request's plain time is its k count times one measured
    plain k point of its bundle and window (every request runs one), and the
    serial latencies replay the arrivals with those durations."""
    import torch

    from aospectrum_b200 import synth
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine
    from aospectrum_b200.kpath import kpath_from_dict
    from aospectrum_b200.serve import BandRequest, BandServer, percentile

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    full = args.stream == "full"
    preset = synth.STREAM_FULL if full else {}
    n_req = args.requests or (6 if full else 12)
    stream = synth.serving_stream(n_req, **preset)
    kpts = kpath_from_dict(synth.ygxm_path(preset.get("path_points", 121))).fractional_points
    bundles, windows = {}, {}
    for r in stream:
        key = r.spec.name
        if key not in bundles:
            bundles[key] = synth.generate_bundle(r.spec)
        wk = (key, r.states)
        if wk not in windows:
            windows[wk] = serving_window(bundles[key], r.states, dev)

    def settings_for(states: int) -> CissSettings:
        # search dimension L*M comfortably above the window's state count
        return CissSettings(block_size=32 if states <= 90 else 64)

    reqs = [BandRequest(bundles[r.spec.name], [kpts[i] for i in r.kpoint_indices],
                        EnergyInterval(*windows[(r.spec.name, r.states)]),
                        settings_for(r.states), f"r{i}") for i, r in enumerate(stream)]
    total_k = sum(len(r.kpoint_indices) for r in stream)
    with ClockSampler(0) as clocks:
        with BandServer(device=dev, slots=4,
                        engine_settings=EngineSettings(precision="mixed")) as srv:
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
    # serial plain baseline: one request at a time, plain complex64 engine
    serial_lat, durations, measured = [], [], {}
    engines = {}
    t0 = time.perf_counter()
    for r, q in zip(stream, reqs):
        key = (r.spec.name, r.states)
        ekey = (r.spec.name, q.settings.block_size)   # the probe block is per engine
        if ekey not in engines:
            for e in engines.values():
                e.close()
            engines = {ekey: BandEngine(q.bundle, q.settings, EngineSettings(precision="plain"),
                                        device=dev)}
        eng = engines[ekey]
        if full:
            if key not in measured:
                eng.solve_kpoints(q.kpoints[:1], q.interval)        # warm
                torch.cuda.synchronize(dev)
                t1 = time.perf_counter()
                eng.solve_kpoints(q.kpoints[1:2] or q.kpoints[:1], q.interval)
                torch.cuda.synchronize(dev)
                measured[key] = time.perf_counter() - t1
            durations.append(measured[key] * len(q.kpoints))
        else:
            now = time.perf_counter() - t0
            if now < r.arrival_s:
                time.sleep(r.arrival_s - now)
            t1 = time.perf_counter()
            eng.solve_kpoints(q.kpoints, q.interval)
            torch.cuda.synchronize(dev)
            durations.append(time.perf_counter() - t1)
            serial_lat.append(time.perf_counter() - t0 - r.arrival_s)
    for e in engines.values():
        e.close()
    if full:
        clock = 0.0
        for r, d in zip(stream, durations):
            clock = max(clock, r.arrival_s) + d
            serial_lat.append(clock - r.arrival_s)
        serial_span = clock
    else:
        serial_span = time.perf_counter() - t0
    lat = [x.latency_seconds for x in responses]
    sizes = [{"atoms": int(np.prod(r.spec.grid)), "orbitals": r.spec.orbitals_per_atom,
              "n": r.spec.n_orbitals, "kpoints": len(r.kpoint_indices), "states": r.states,
              "block_size": settings_for(r.states).block_size,
              "arrival_s": round(r.arrival_s, 3)} for r in stream]
    desc = ("c4 serving stream at the specified sizes: first %d requests of the seeded stream "
            "(216-8000-atom cubic bundles, 5 or 13 orbitals, 16-256 k points from a 301-point "
            "Y-G-X-M path, windows of 20-200 Gamma states), Poisson arrivals at 2/s" % n_req
            if full else
            "c4 serving stream, reduced sizes: 12 requests, 216-1000-atom cubic bundles, 5 or "
            "13 orbitals, 4-16 k points, windows of 20-60 Gamma states, Poisson arrivals at 2/s")
    out = {"metric": "serving k-points/s with p50/p99 latency (continuous batching, 1 B200)",
           "value": total_k / span, "unit": "k-points/s", "n_gpus": 1, "steps": 1, "warmup": 0,
           "ms_per_step": span * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c64+bf16x3 tensor-core updates, fp64 refinement",
           "data": "synthetic (seeded serving stream)",
           "config": {"workload": desc, "requests": len(stream), "kpoints": total_k, "slots": 4,
                      "bundles": sorted({r.spec.name for r in stream}), "sizes": sizes},
           "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
           "server_stats": stats, "clocks": clocks.summary(),
           "serial_plain": {"kpoints_per_s": total_k / serial_span,
                            "p50_latency_s": percentile(serial_lat, 50),
                            "p99_latency_s": percentile(serial_lat, 99),
                            "method": ("each request's duration = its k count x one measured "
                                       "plain k point of its bundle and window; arrivals "
                                       "replayed" if full else
                                       "every request solved, arrivals replayed")},
           "max_residual_ev": max(x.maximum_residual_ev for x in responses)}
    print(json.dumps(out), flush=True)


def sweep_indices(spec: str, count: int) -> list[int]:
    if spec == "all":
        return list(range(count))
    if ":" in spec:
        a, b, s = (int(v) if v else None for v in (spec.split(":") + [""])[:3])
        return list(range(count))[slice(a, b, s)]
    return [int(v) for v in spec.split(",")]


def match_errors(got: np.ndarray, exact: np.ndarray) -> tuple[float, int]:
    """Max |E - E_FP64| over the FP64 eigenvalues matched in sorted order
    (the larger set is trimmed at whichever end matches better), and the
    count difference."""
    got = np.sort(np.asarray(got, np.float64))
    exact = np.sort(np.asarray(exact, np.float64))
    if got.size == 0 or exact.size == 0:
        return 0.0, int(got.size - exact.size)
    m = min(got.size, exact.size)
    best = float("inf")
    big, small = (got, exact) if got.size >= exact.size else (exact, got)
    for off in range(big.size - m + 1):
        best = min(best, float(np.max(np.abs(big[off:off + m] - small))))
    return best, int(got.size - exact.size)


def accuracy_sweep(args) -> None:
    """Per-k accuracy record: the mixed (chosen) and plain complex64 forms
    at the same k points, each against FP64 dense generalized eigenvalues
    of the same H(k), S(k), with the max eigenpair residuals of both."""
    import torch

    from aospectrum_b200 import synth
    from aospectrum_b200.ciss import CissSettings, EngineSettings
    from aospectrum_b200.data import EnergyInterval
    from aospectrum_b200.engine import BandEngine

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    w, kp = workload(args.workload)
    bundle = synth.generate_bundle(w.spec)
    interval = EnergyInterval(w.window_ev[0] - GUARD_EV, w.window_ev[1] + GUARD_EV)
    settings = CissSettings(integration_points=w.integration_points, block_size=w.block_size,
                            moment_size=w.moment_size)
    kpts = kp.fractional_points
    idx = sweep_indices(args.accuracy_sweep, len(kpts))
    mixed = BandEngine(bundle, settings, EngineSettings(
        precision="mixed", ordering=args.ordering,
        **({"refinement_steps": args.refinement_steps} if args.refinement_steps >= 0 else {})),
        device=dev)
    plain = BandEngine(bundle, settings, EngineSettings(precision="plain", ordering=args.ordering),
                       device=dev) if args.plain_kpoints > 0 else None
    rows = []
    t0 = time.perf_counter()
    for i in idx:
        k = kpts[i]
        rm, _ = mixed.solve_kpoints([k], interval)
        row = {"k_index": i, "k": [float(v) for v in k],
               "mixed_count": int(rm[0].energies_ev.size),
               "mixed_residual_ev": rm[0].maximum_residual_ev}
        if plain is not None:
            rp, _ = plain.solve_kpoints([k], interval)
            row["plain_count"] = int(rp[0].energies_ev.size)
            row["plain_residual_ev"] = rp[0].maximum_residual_ev
            row["mixed_vs_plain_ev"], _ = match_errors(rm[0].energies_ev, rp[0].energies_ev)
        exact = fp64_window(mixed.host_pair(k), interval, dev)
        row["fp64_count"] = int(exact.size)
        row["mixed_error_ev"], row["mixed_count_diff"] = match_errors(rm[0].energies_ev, exact)
        if plain is not None:
            row["plain_error_ev"], row["plain_count_diff"] = match_errors(rp[0].energies_ev, exact)
        edge = np.min(np.abs(np.concatenate([exact - interval.lower_ev,
                                             interval.upper_ev - exact]))) if exact.size else None
        row["fp64_nearest_edge_ev"] = float(edge) if edge is not None else None
        rows.append(row)
        print(json.dumps(row), flush=True)
    mixed.close()
    if plain is not None:
        plain.close()

    def worst(key):
        vals = [r[key] for r in rows if key in r]
        return max(vals) if vals else None

    out = {"workload": f"{w.name}: {w.notes}", "kpoints": len(rows),
           "interval_ev": [interval.lower_ev, interval.upper_ev],
           "oracle": "FP64 dense generalized eigh (torch, cuSOLVER) of the same H(k), S(k)",
           "max_mixed_error_ev": worst("mixed_error_ev"),
           "max_plain_error_ev": worst("plain_error_ev"),
           "max_mixed_residual_ev": worst("mixed_residual_ev"),
           "max_plain_residual_ev": worst("plain_residual_ev"),
           "max_mixed_vs_plain_ev": worst("mixed_vs_plain_ev"),
           "count_mismatches_mixed": sum(1 for r in rows if r["mixed_count_diff"]),
           "count_mismatches_plain": sum(1 for r in rows if r.get("plain_count_diff")),
           "seconds": time.perf_counter() - t0, "per_k": rows}
    if args.sweep_out:
        Path(args.sweep_out).write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps({k: v for k, v in out.items() if k != "per_k"}), flush=True)


def main() -> None:
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.workload == "c4":
        serving_arm(args)
        return
    if args.accuracy_sweep:
        accuracy_sweep(args)
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
    if args.schur_pairs >= 0:
        native.library().aosb_factor_set_schur_pairs(args.schur_pairs)
    if args.solve_lookahead >= 0:
        native.library().aosb_solve_set_lookahead(args.solve_lookahead)
    look_on = native.library().aosb_solve_set_lookahead(0)
    native.library().aosb_solve_set_lookahead(look_on)
    pairs_on = native.library().aosb_factor_set_schur_pairs(0)
    native.library().aosb_factor_set_schur_pairs(pairs_on)
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
                                       if args.tensor_core_solves >= 0 else {}),
                                    **({"cuda_graphs": bool(args.cuda_graphs)}
                                       if args.cuda_graphs >= 0 else {})), device=dev)
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
        # algorithmic complex flops (8 per complex FMA) against the full
        # sustained BF16 peak: the split-BF16 hi/lo products are overhead,
        # not work; their issue rate is reported beside it
        sustained = peaks.get("bf16_tflops_sustained")
        peak = sustained if sustained else 1400.0
        achieved = k_flops.value / (k_ms.value / 1e3) / 1e12
        per_launch_units = k_flops.value / k_launches.value / (8.0 * info.tile ** 3)
        traffic = schur_traffic_per_unit()
        roofline = {
            "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak,
            "traffic": traffic["bytes_per_unit"] * per_launch_units if traffic else None,
            "traffic_source": traffic["source"] if traffic else None,
            "kernel": "schur_tc_kernel",
            "launches": int(k_launches.value),
            "avg_launch_ms": k_ms.value / k_launches.value,
            "algorithmic_flops_per_launch": k_flops.value / k_launches.value,
            "algorithmic_bytes_per_launch": k_bytes.value / k_launches.value,
            "achieved_hbm_gbs": k_bytes.value / (k_ms.value / 1e3) / 1e9,
            "hbm_peak_gbs": peaks.get("hbm_gbs", 6650.0),
            "split_bf16_issue_frac": 3.0 * achieved / peak,
            "peak_source": ("of measured: MEASURED_PEAKS.json bf16_tflops_sustained"
                            if sustained else "of fallback: 1400 TFLOP/s sustained"),
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
                   "cuda_graphs": bool(eng.engine.cuda_graphs),
                   "schur_depth": eng.engine.schur_depth,
                   "schur_pairs": bool(pairs_on),
                   "solve_lookahead": bool(look_on),
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
        checks = []
        if not dense_ok and args.fp64_check > 0:
            from aospectrum_b200.fp64check import fp64_check

            check_iv = (EnergyInterval(*w.window_ev) if args.fp64_check_interval == "window"
                        else interval)
            for i in range(min(args.fp64_check, len(kpts))):
                kpt = kpts[(i * 37) % len(kpts)]
                try:
                    c = fp64_check(eng, kpt, check_iv)
                except Exception as exc:   # the timed result above still gets printed
                    c = {"error": f"{type(exc).__name__}: {exc}"[:300]}
                    torch.cuda.empty_cache()
                c["interval_ev"] = [check_iv.lower_ev, check_iv.upper_ev]
                c["k_index"] = (i * 37) % len(kpts)
                checks.append(c)
                errs.append(c["max_eig_error_ev"] if c.get("max_eig_error_ev") is not None
                            else float("inf"))
        out["accuracy"] = {"max_eig_error_ev": max(errs) if errs else None,
                           "kpoints_checked": len(errs),
                           "max_residual_ev": max(r.maximum_residual_ev for rs in results
                                                  for r in rs),
                           # k points whose CISS search space (L x M columns) saturated:
                           # the interval holds more states than it can resolve
                           "saturated_kpoints": sum(1 for rs in results for r in rs
                                                    if not r.complete),
                           "search_dimension": w.block_size * w.moment_size,
                           "oracle": ("FP64 dense generalized eigh (torch, cuSOLVER) of the "
                                      "same H(k), S(k)" if dense_ok else
                                      "FP64 refinement (aospectrum_b200.fp64check): one "
                                      "shift-invert step per eigenpair with solves refined in "
                                      "FP64 to 1e-9 relative, FP64 Rayleigh-Ritz, residual/gap "
                                      "bound of the refined values")}
        if checks:
            out["accuracy"]["fp64_check"] = checks
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
        if world == 1:
            out["ingest"] = ingest_leg(bundle, dev)
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(bundle, [kpts[0]], interval.lower_ev,
                                               interval.upper_ev, w)
        print(json.dumps(out), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


def schur_traffic_per_unit() -> dict | None:
    """DRAM bytes per algorithmic unit of schur_tc_kernel -- one (target
    tile, tile step, pencil) update, 8 T^3 flops -- from the committed ncu
    capture summary of the two-step kernel (dram__bytes_read.sum +
    write.sum of the captured launch divided by the units it applied)."""
    f = ROOT / "profiles" / "schur_tc_kernel_two_step_c2.json"
    if not f.exists():
        return None
    d = json.loads(f.read_text())
    return {"bytes_per_unit": float(d["dram_bytes_per_unit"]),
            "source": f"profiles/{f.name}: {d['workload']}"}


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


def ingest_leg(bundle, dev) -> dict:
    """Bundle ingest on this box: the bundle is written to a
    temporary directory (untimed), then opened memory-mapped (load_bundle),
    its CSR pattern and Bloch tables built by the C++ host code
    (aosb_bloch_create), the block values copied from the memory map into
    pinned host memory and from there to the device."""
    import tempfile

    import torch

    from aospectrum_b200.bundle import load_bundle, write_bundle
    from aospectrum_b200.engine import BlochDevice

    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        root = Path(tmp) / "bundle"
        write_bundle(bundle, root)
        t0 = time.perf_counter()
        loaded = load_bundle(root)
        out["open_memmap_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        bd = BlochDevice(loaded, dev, upload=False)
        out["pattern_build_cpp_s"] = time.perf_counter() - t0
        ops = loaded.operators
        nbytes = 0
        t0 = time.perf_counter()
        pinned = []
        for arr in (ops.h_values, ops.s_values):
            a = np.asarray(arr)
            t = torch.empty(a.shape, dtype=torch.from_numpy(a[:1].copy()).dtype, pin_memory=True)
            t.numpy()[...] = a
            pinned.append(t)
            nbytes += a.nbytes
        out["memmap_to_pinned_s"] = time.perf_counter() - t0
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        dev_copies = [t.to(dev, non_blocking=True) for t in pinned]
        torch.cuda.synchronize(dev)
        out["pinned_to_device_s"] = time.perf_counter() - t0
        out["value_bytes"] = nbytes
        out["pinned_to_device_gbs"] = nbytes / out["pinned_to_device_s"] / 1e9
        t0 = time.perf_counter()
        bd.upload()
        torch.cuda.synchronize(dev)
        out["tables_and_values_upload_s"] = time.perf_counter() - t0
        bd.close()
        del dev_copies, pinned, loaded
    return {k: (round(v, 4) if isinstance(v, float) else v) for k, v in out.items()}


def e2e_leg(eng, bundle, kset, interval, args) -> dict:
    """Public-API path with host buffers: every step copies the bundle's
    block values from pinned host memory into the engine and reads the
    energies back."""
    import torch

    hv = torch.from_numpy(np.array(bundle.operators.h_values)).pin_memory()
    sv = torch.from_numpy(np.array(bundle.operators.s_values)).pin_memory()
    # at most 20 steps: on the large workloads the timed region already
    # covers every k point of the path, and this leg repeats the same work
    steps = max(1, min(args.steps, 20))
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
