#!/usr/bin/env python
"""Benchmark of the exact clustering trees (headline: HDBSCAN 1,000,000 x 8).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload hdbscan|single32|c1|ward|c4|batch]

Workloads (synthetic data of the configurations' shapes; no public data set
stands behind them):
  hdbscan   (default) HDBSCAN min_samples 25 on 1,000,000 x 8: 20 isotropic
            Gaussian blobs (centres uniform in [-10, 10]^8, std 1, 45,000
            points each) plus 100,000 points uniform over their bounding box,
            float32, shuffled, seed 1. One step = one full exact tree: core
            distances (k = 25), Borůvka MST of mutual reachability, sorted
            merges, scipy-format Z and the core distances on the host.
  single32  single linkage on 1,000,000 x 32 standard normal, seed 0.
  c1        single linkage on 20,000 x 32 standard normal, seed 0.
  ward      Ward (RNN rounds) on 1,000,000 x 32 standard normal, seed 2.
  c4        single linkage on 4,000,000 x 16: 50 Gaussian clusters, each with
            its own random covariance (eigenvalues log-uniform in [0.05, 5]),
            plus 5% uniform noise, seed 3; screened, screened + learned radius
            proposal, plain.
  batch     4,096 mixed single-linkage / HDBSCAN instances (n 64-50k, d 2/8/32).

Prints one JSON line (rank 0). For the tree workloads `value` is the
device-resident time per tree (points already in HBM, the *_device entry
points); `e2e` is the same through the host API (cuhc_hdbscan_tree /
cuhc_linkage) with pinned host buffers, copies included. `--impl reference`
runs the reference library (shangar21/cuhc built from its sources for
sm_100a, oracle/_ref/libcuhc.so) through its own C ABI with host buffers and
its default pruning, on the same data and GPU, and prints the same `config`.
With N > 1 GPUs each rank builds its own tree (replicas; the path does not
shard).

Outside the timed region the line also carries: the same step with the
tensor-core screen off (`plain_fp32`) and whether its tree is bit-identical
(`parity.identical_to_plain`); one audited step (`screen_audit`: every
evaluated pair's screened value against the FP32 and FP64 distances); and,
in the CPU-baseline leg, scikit-learn / scipy timed on the host cores, with
the oracle (sampled core distances) and the reference library (pruning off,
its bit-parity mode) as checkers of the step's tree.
"""

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
METRIC = "1M-pt single/HDBSCAN MST time (s) on 1 B200, screened vs plain FP32, exact tree"
UNIT = "s"
N_POINTS, N_FEATURES, MIN_SAMPLES = 1_000_000, 8, 25
L2_FLUSH_BYTES = 256 << 20
SM_COUNT = 148

f32p, f64p = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)


# ---------------------------------------------------------------------------
# Data

def make_blobs_with_noise(seed=1, n=N_POINTS, d=N_FEATURES, centers=20, noise=0.10):
    """The headline data set: equal Gaussian blobs (std 1) + uniform noise."""
    rng = np.random.default_rng(seed)
    n_noise = int(round(n * noise))
    per = (n - n_noise) // centers
    centres = rng.uniform(-10.0, 10.0, (centers, d))
    pts = np.repeat(centres, per, axis=0) + rng.standard_normal((per * centers, d))
    lo, hi = pts.min(axis=0), pts.max(axis=0)
    X = np.vstack([pts, rng.uniform(lo, hi, (n - per * centers, d))]).astype(np.float32)
    return np.ascontiguousarray(X[rng.permutation(len(X))])


def make_batch_instances(count=4096, seed=4):
    """The batched workload: `count` problems, n = round(exp(U(ln 64, ln 50,000))),
    d uniform in {2, 8, 32}, 1-12 Gaussian blobs (centres U[-10, 10]^d, std
    U(0.5, 2.0)) plus 5% uniform noise over their bounding box, float32;
    alternately single linkage (min_samples 0) and HDBSCAN (min_cluster_size
    10, so min_samples 10)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(64), np.log(50_000)))))
        d = int(rng.choice([2, 8, 32]))
        blobs = int(rng.integers(1, 13))
        n_noise = int(round(0.05 * n))
        m = n - n_noise
        centres = rng.uniform(-10.0, 10.0, (blobs, d))
        stds = rng.uniform(0.5, 2.0, blobs)
        label = rng.integers(0, blobs, m)
        pts = centres[label] + rng.standard_normal((m, d)) * stds[label, None]
        lo, hi = pts.min(axis=0), pts.max(axis=0)
        X = np.vstack([pts, rng.uniform(lo, hi, (n_noise, d))]).astype(np.float32)
        out.append((np.ascontiguousarray(X[rng.permutation(n)]), 0 if i % 2 == 0 else 10))
    return out


# Tree workloads: data, (linkage id, algorithm id) of cuhc_linkage, label.
TREES = {
    "single32": dict(n=1_000_000, d=32, seed=0, linkage=0, algorithm=1,
                     label="single linkage (Borůvka)",
                     recipe="1,000,000 x 32 standard normal, seed 0"),
    "c1": dict(n=20_000, d=32, seed=0, linkage=0, algorithm=1, label="single linkage (Borůvka)",
               recipe="20,000 x 32 standard normal, seed 0"),
    "ward": dict(n=1_000_000, d=32, seed=2, linkage=3, algorithm=3, label="Ward (RNN rounds)",
                 recipe="1,000,000 x 32 standard normal, seed 2"),
    "c4": dict(n=4_000_000, d=16, seed=3, linkage=0, algorithm=1, label="single linkage (Borůvka)",
               recipe="4,000,000 x 16: 50 Gaussian clusters, each with its own random "
                      "covariance (eigenvalues log-uniform in [0.05, 5]), + 5% noise, seed 3"),
}


def tree_data(workload, n=None):
    spec = TREES[workload]
    n = n or spec["n"]
    if workload == "c4":
        sys.path.insert(0, HERE)
        from cuhc_b200.train_radius import make_anisotropic_blobs  # noqa: PLC0415
        return make_anisotropic_blobs(spec["seed"], n)
    return np.random.default_rng(spec["seed"]).standard_normal((n, spec["d"])).astype(np.float32)


def workload_config(workload, n, d):
    """The `config` both arms print for a workload (identical keys)."""
    if workload == "hdbscan":
        return {"workload": f"hdbscan {n:,} x {d}, 20 blobs + 10% noise, min_samples 25",
                "n": n, "d": d, "min_samples": MIN_SAMPLES}
    spec = TREES[workload]
    return {"workload": f"{spec['label']}: {spec['recipe']}" if n == spec["n"] else
            f"{spec['label']}: {n:,} points of the recipe {spec['recipe']}", "n": n, "d": d}


# ---------------------------------------------------------------------------
# Measurement helpers

class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.proc, self.file = gpu, None, None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.file:
            return None
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        max_mhz = float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": float(np.median(loaded)) if loaded else None,
                "sm_max_mhz": max_mhz, "reasons": reasons, "samples": len(rows)}


def fp32_peak_tflops(torch):
    """Measured FP32 (non-tensor) throughput: cuBLAS SGEMM 8192^3, TF32 off."""
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(8192, 8192, device="cuda")
    b = torch.randn(8192, 8192, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2 * 8192 ** 3 / best / 1e12


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def chunk_width(d):
    return 4 if d <= 4 else 8 if d <= 8 else 16 if d <= 16 else 32


def roofline(kt, d, fp32, clocks):
    """Roofline of the dominant pass kind (the one with the most device time),
    timed with CUDA events on its own stream inside the library."""
    peaks, peak_kind = measured_peaks()
    kind, (ms, launches, tiles) = max(kt.items(), key=lambda kv: kv[1][0])
    pairs = tiles * 128 * 128
    seconds = ms / 1e3
    sgemm = f"cuBLAS SGEMM 8192^3 with TF32 off, measured in this run: {fp32:.2f} TFLOP/s"
    sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
    per_sm_cycle = pairs / (seconds * sm_mhz * 1e6 * SM_COUNT) if seconds > 0 else 0.0
    if kind.startswith("screen"):
        # 2d tensor FLOP per evaluated pair (the -2 X Y^T product) against the
        # TF32 rate, half the measured bf16 burst. The MMAs issue K = KC + 8
        # (coordinates padded to the chunk width, four norm terms, at least
        # four component slots).
        peak = peaks["bf16_tflops"] / 2 if peaks.get("bf16_tflops") else None
        achieved = pairs * 2 * d / seconds / 1e12 if seconds > 0 else 0.0
        k_pad = (chunk_width(d) + 8 + 7) // 8 * 8
        issued = pairs * 2 * k_pad / seconds / 1e12 if seconds > 0 else 0.0
        return {"bound": "tensor", "kernel": kind, "achieved": round(achieved, 2),
                "peak": round(peak, 1) if peak else None, "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4) if peak else None, "traffic": None,
                "peak_source": f"TF32 = half the bf16 burst {peaks.get('bf16_tflops')} "
                               f"TFLOP/s ({peak_kind})",
                "work": f"{tiles} tiles x 16384 pairs x 2d FLOP in {launches} launches, "
                        f"{ms:.1f} ms",
                "issued_tflops": round(issued, 2), "issued_k": k_pad,
                "pairs_per_sm_cycle": {
                    "achieved": round(per_sm_cycle, 2), "sm_mhz": sm_mhz,
                    "tensor_ceiling": round(4096 / (2 * k_pad), 1),
                    "epilogue_issue_ceiling": 256,
                    "note": "tensor: 4096 TF32 FLOP per SM-cycle / 2K; epilogue: 4 warp "
                            "instructions per SM-cycle, each a 3-input min over 64 pairs"},
                "fp32_equivalent": {"achieved": round(pairs * 3 * d / seconds / 1e12, 2),
                                    "peak": round(fp32, 2), "peak_source": sgemm}}
    achieved = pairs * 3 * d / seconds / 1e12 if seconds > 0 else 0.0
    return {"bound": "fp32", "kernel": kind, "achieved": round(achieved, 2),
            "peak": round(fp32, 2), "unit": "TFLOP/s",
            "frac": round(achieved / fp32, 3) if fp32 else None, "traffic": None,
            "peak_source": sgemm,
            "work": f"{tiles} tiles x 16384 pairs x 3d FLOP in {launches} launches, {ms:.1f} ms",
            "pairs_per_sm_cycle": {"achieved": round(per_sm_cycle, 2), "sm_mhz": sm_mhz}}


def passes_summary(kt, sc, tiles_per_step=None, rounds_per_step=None):
    out = {k: {"ms": round(v[0], 2), "launches": v[1], "tiles": v[2]} for k, v in kt.items()}
    screened_tiles = sum(v[2] for k, v in kt.items() if k.startswith("screen"))
    out["screen"] = {**sc, "rechecks_per_pair": round(sc["rechecks"] / max(1, 16384 * screened_tiles),
                                                      6)}
    if tiles_per_step is not None:
        out["tiles_per_step"] = tiles_per_step
        out["rounds_per_step"] = rounds_per_step
    return out


def audit_summary(audit):
    """The screen audit of one step, rounded for the JSON line."""
    def r(x):
        return None if x is None or x != x else float(f"{x:.4g}")
    return {"pairs": audit["pairs"], "violations": audit["violations"],
            "min_slack": r(audit["min_slack"]),
            "screened_bound_vs_fp64": {"max_abs": r(audit["max_bound_gap_abs"]),
                                       "max_rel_to_norms": r(audit["max_bound_gap_rel_norms"])},
            "exact_fp32_vs_fp64": {"max_abs": r(audit["max_exact_abs"]),
                                   "max_rel": r(audit["max_exact_rel"])},
            "note": "every evaluated pair of one step: screened lower bound D' vs the reference "
                    "FP32 squared distance s (violations = D' > s, must be 0; slack = "
                    "(s - D') / (e (|x|^2 + |y|^2)), >= 0 required, ~0.5+ = modelled error "
                    "bound holds with room) and both vs an FP64 recomputation"}


# ---------------------------------------------------------------------------
# CPU baseline and checkers (the only part of the arm that runs oracle/ code,
# after every timed region)

def sklearn_hdbscan_baseline(n_sample, ours_time):
    """scikit-learn's HDBSCAN (the reference's own test oracle) fitted on
    n_sample points of the headline recipe, on every host core."""
    from sklearn.cluster import HDBSCAN  # noqa: PLC0415
    X = make_blobs_with_noise(n=n_sample)
    t0 = time.perf_counter()
    HDBSCAN(min_cluster_size=MIN_SAMPLES, min_samples=MIN_SAMPLES, n_jobs=-1, copy=True).fit(X)
    elapsed = time.perf_counter() - t0
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return {"value": round(elapsed, 3), "unit": UNIT, "cores": cores, "kind": "sklearn",
            "sample": f"sklearn.cluster.HDBSCAN(min_cluster_size=25, min_samples=25, n_jobs=-1) "
                      f"fit on {n_sample:,} points of the same recipe (seed 1), timed once",
            "n": n_sample, "ours_same_n_s": round(ours_time, 4),
            "scaled_to_workload_s": round(elapsed * (N_POINTS / n_sample) ** 2, 1),
            "scaling_note": "quadratic in n (its Prim MST over mutual reachability)"}


def scipy_single_baseline(X, n_sample, ours_time):
    from scipy.cluster.hierarchy import linkage  # noqa: PLC0415
    Y = X[:n_sample]
    t0 = time.perf_counter()
    linkage(Y, "single")
    elapsed = time.perf_counter() - t0
    return {"value": round(elapsed, 3), "unit": UNIT, "cores": 1, "kind": "scipy",
            "sample": f"scipy.cluster.hierarchy.linkage(X[:{n_sample}], 'single') "
                      f"(single-threaded), timed once", "n": n_sample,
            "ours_same_n_s": None if ours_time is None else round(ours_time, 4),
            "scaled_to_workload_s": round(elapsed * (len(X) / n_sample) ** 2, 1)}


def sklearn_ward_baseline(X, n_sample, ours_time):
    from sklearn.cluster import AgglomerativeClustering  # noqa: PLC0415
    Y = X[:n_sample]
    t0 = time.perf_counter()
    AgglomerativeClustering(n_clusters=1, linkage="ward", compute_full_tree=True).fit(Y)
    elapsed = time.perf_counter() - t0
    return {"value": round(elapsed, 3), "unit": UNIT, "cores": 1, "kind": "sklearn",
            "sample": f"sklearn AgglomerativeClustering(linkage='ward') on X[:{n_sample}] "
                      f"(n^2 memory: 1M points would need 4 TB), timed once", "n": n_sample,
            "ours_same_n_s": None if ours_time is None else round(ours_time, 4)}


def reference_checks(X, tree, core=None, linkage=None, min_samples=None, oracle_rows=2000):
    """The step's tree against the checkers: the reference library with
    pruning off (its bit-parity mode) and, for HDBSCAN, the C oracle's core
    distances on sampled rows."""
    sys.path.insert(0, HERE)
    from oracle import oracle as O  # noqa: PLC0415
    out = {}
    if core is not None and oracle_rows:
        # The data are shuffled, so the first rows are a random sample.
        O.set_threads(os.cpu_count() or 1)
        ref_core = O.core_distances(X, min_samples, rows=(0, oracle_rows))
        out["oracle_core_rows_identical"] = bool(np.array_equal(ref_core, core[:oracle_rows]))
        out["oracle_core_rows"] = oracle_rows
    if O.reference_available():
        t0 = time.perf_counter()
        if min_samples is not None:
            Z_ref, core_ref = O.reference_hdbscan_tree(X, min_samples, pruning="never")
            out["reference_core_identical"] = bool(np.array_equal(core_ref, core))
        else:
            method, algorithm = linkage
            Z_ref = O.reference_linkage(X, method, algorithm, pruning="never")
        out["reference_tree_identical"] = bool(np.array_equal(Z_ref.ravel(), tree.ravel()))
        out["reference_s"] = round(time.perf_counter() - t0, 2)
        out["reference_mode"] = "oracle/_ref (reference built from source), pruning never"
    return out


# ---------------------------------------------------------------------------
# Our arm: the headline HDBSCAN tree

def run_hdbscan(args, rank, world, local_rank):
    import torch  # noqa: PLC0415
    import torch.distributed as dist  # noqa: PLC0415
    sys.path.insert(0, HERE)
    from cuhc_b200 import _lib  # noqa: PLC0415

    X = make_blobs_with_noise(n=args.n or N_POINTS)
    n, d = X.shape
    X_dev = torch.from_numpy(X).cuda()
    X_pin = torch.from_numpy(X).pin_memory()
    tree_pin = torch.empty((n - 1) * 4, dtype=torch.float64).pin_memory()
    core_pin = torch.empty(n, dtype=torch.float32).pin_memory()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    tree_ptr = ctypes.cast(tree_pin.data_ptr(), f64p)
    core_ptr = ctypes.cast(core_pin.data_ptr(), f32p)

    def device_step():
        _lib.check(_lib.lib.cuhc_hdbscan_tree_device(
            ctypes.c_void_p(X_dev.data_ptr()), n, d, 0, 2.0, MIN_SAMPLES, 1.0, 0, tree_ptr,
            core_ptr))

    def host_step():
        _lib.check(_lib.lib.cuhc_hdbscan_tree(
            ctypes.cast(X_pin.data_ptr(), f32p), n, d, 0, 2.0, MIN_SAMPLES, 1.0, 0, tree_ptr,
            core_ptr))

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def timed(step, k):
        """Device time per step (CUDA events; L2 flushed before each step)."""
        times = []
        for _ in range(k):
            flush.zero_()
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            step()
            e.record()
            e.synchronize()
            times.append(s.elapsed_time(e) / 1e3)
        return times

    for _ in range(args.warmup):
        device_step()
    barrier()
    launches0 = _lib.launch_count()
    stats0 = _lib.pass_stats()
    with ClockSampler(local_rank) as clocks:
        barrier()
        times = timed(device_step, args.steps)
        barrier()
    launches = (_lib.launch_count() - launches0) // max(args.steps, 1)
    stats1 = _lib.pass_stats()
    per_step = float(np.mean(times))
    screened_tree = tree_pin.numpy().copy()
    screened_core = core_pin.numpy().copy()

    # Kernel-level figures: the pass kernels timed on their own stream.
    _lib.set_timing(True)
    _lib.kernel_timing()
    _lib.screen_counters()
    timed(device_step, 1)
    kt = _lib.kernel_timing()
    sc = _lib.screen_counters()
    _lib.set_timing(False)

    # The same step with tensor-core screening switched off (plain FP32 passes).
    plain, identical_plain = float("nan"), None
    if not args.no_plain:
        _lib.set_screen("off")
        device_step()
        plain = float(np.mean(timed(device_step, max(1, min(args.steps, 3)))))
        identical_plain = bool(np.array_equal(tree_pin.numpy(), screened_tree) and
                               np.array_equal(core_pin.numpy(), screened_core))
        _lib.set_screen("auto")

    # End to end through the host API (pinned buffers, copies included).
    host_step()
    e2e_times = timed(host_step, args.steps)
    e2e = float(np.mean(e2e_times))
    identical_e2e = bool(np.array_equal(tree_pin.numpy(), screened_tree))

    # One audited step: every evaluated pair's screened bound against FP32 / FP64.
    _lib.set_screen_audit(True)
    _lib.screen_audit()
    device_step()
    audit = _lib.screen_audit()
    _lib.set_screen_audit(False)
    identical_audited = bool(np.array_equal(tree_pin.numpy(), screened_tree))

    t = torch.tensor([per_step, e2e, plain], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    per_step, e2e, plain = float(t[0]), float(t[1]), float(t[2])

    if rank == 0:
        clock = clocks.summary()
        fp32 = fp32_peak_tflops(torch)
        line = {
            "metric": METRIC, "value": round(per_step, 4), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 2),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": workload_config("hdbscan", n, d),
            "setup": {"path": "tcgen05 TF32 screen + exact FP32 recheck",
                      "l2": "flushed before every step (256 MB write)",
                      "parallelism": f"replicas x{world}",
                      "knn_pipeline_shape": dict(zip(("stages", "lead"), _lib.screen_shape()),
                                                 chosen_by="shape tuner, first call")},
            "e2e": {"value": round(e2e, 4), "unit": UNIT, "h2d_bytes_per_step": int(X.nbytes),
                    "d2h_bytes_per_step": int((n - 1) * 4 * 8 + n * 4)},
            "gpu_launches": int(launches),
            "step_ms": {"device": [round(x * 1e3, 2) for x in times],
                        "e2e": [round(x * 1e3, 2) for x in e2e_times]},
            "roofline": roofline(kt, d, fp32, clock),
            "plain_fp32": {"value": None if np.isnan(plain) else round(plain, 4), "unit": UNIT,
                           "speedup_screened": None if np.isnan(plain) else
                           round(plain / per_step, 2),
                           "note": "same step with tensor-core screening off"},
            "parity": {"identical_to_plain": identical_plain,
                       "e2e_identical": identical_e2e, "audited_identical": identical_audited},
            "screen_audit": audit_summary(audit),
            "passes": passes_summary(kt, sc, int((stats1[0] - stats0[0]) / max(args.steps, 1)),
                                     (stats1[3] - stats0[3]) / max(args.steps, 1)),
            "clocks": clock,
        }
        if world == 1 and not args.no_cpu_baseline:
            small = make_blobs_with_noise(n=args.cpu_sample)
            small_tree = np.empty((len(small) - 1) * 4, np.float64)
            small_core = np.empty(len(small), np.float32)
            small_dev = torch.from_numpy(small).cuda()

            def small_step():
                _lib.check(_lib.lib.cuhc_hdbscan_tree_device(
                    ctypes.c_void_p(small_dev.data_ptr()), len(small), d, 0, 2.0, MIN_SAMPLES,
                    1.0, 0, small_tree.ctypes.data_as(f64p), small_core.ctypes.data_as(f32p)))
            small_step()
            ours_small = float(np.mean(timed(small_step, 3)))
            line["cpu_baseline"] = sklearn_hdbscan_baseline(args.cpu_sample, ours_small)
            if not args.no_parity:
                line["parity"].update(reference_checks(
                    X, screened_tree, screened_core, min_samples=MIN_SAMPLES))
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Our arm: single-linkage / Ward trees

def run_tree_workload(args, local_rank):
    """Device-resident time per tree through cuhc_linkage_device for each
    variant (screened; c4 also with the learned radius proposal; plain FP32),
    with the trees compared bit for bit."""
    import torch  # noqa: PLC0415
    sys.path.insert(0, HERE)
    import cuhc_b200 as C  # noqa: PLC0415
    from cuhc_b200 import _lib  # noqa: PLC0415
    spec = TREES[args.workload]
    X = tree_data(args.workload, args.n)
    n, d = X.shape
    dev = torch.from_numpy(X).cuda()
    X_pin = torch.from_numpy(X).pin_memory()
    tree = np.empty((n - 1) * 4, np.float64)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def step():
        _lib.check(_lib.lib.cuhc_linkage_device(ctypes.c_void_p(dev.data_ptr()), n, d, 0, 2.0,
                                                spec["linkage"], spec["algorithm"],
                                                tree.ctypes.data_as(f64p)))

    def host_step():
        _lib.check(_lib.lib.cuhc_linkage(ctypes.cast(X_pin.data_ptr(), f32p), n, d, 0, 2.0,
                                         spec["linkage"], spec["algorithm"],
                                         tree.ctypes.data_as(f64p)))

    def timed(fn, k):
        times = []
        for _ in range(k):
            flush.zero_()
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            e.synchronize()
            times.append(s.elapsed_time(e) / 1e3)
        return float(np.mean(times))

    variants = [("screened", "auto", False)]
    if args.workload == "c4":
        variants.append(("screened + radius proposal", "auto", True))
    if not args.no_plain:
        variants.append(("plain fp32", "off", False))
    results, screened_tree, kt, sc = {}, None, None, None
    launches = None
    with ClockSampler(local_rank) as clocks:
        for name, screen, radius in variants:
            _lib.set_screen(screen)
            if radius:
                meta = C.load_radius_model()
            for _ in range(args.warmup):
                step()
            C.radius_stats()
            launches0 = _lib.launch_count()
            t = timed(step, args.steps)
            if name == "screened":
                launches = (_lib.launch_count() - launches0) // max(args.steps, 1)
            stats = C.radius_stats()
            results[name] = {"s": round(t, 4)}
            if radius:
                results[name]["certified_share"] = round(
                    stats["certified"] / max(1, stats["proposed"]), 4)
                results[name]["tiles_per_tree"] = {
                    "capped_passes": stats["capped_tiles"] // max(1, args.steps),
                    "fallback_passes": stats["fallback_tiles"] // max(1, args.steps)}
                results[name]["model"] = (f"trained on seeds {list(meta['seeds'])}, n = "
                                          f"{int(meta['n'])}, {int(meta['rows'])} rows")
                C.set_radius_model(None)
            if screened_tree is None:
                screened_tree = tree.copy()
                _lib.set_timing(True)
                _lib.kernel_timing()
                _lib.screen_counters()
                timed(step, 1)
                kt, sc = _lib.kernel_timing(), _lib.screen_counters()
                _lib.set_timing(False)
            results[name]["identical_to_screened"] = bool(np.array_equal(tree, screened_tree))
    _lib.set_screen("auto")
    host_step()
    e2e = timed(host_step, max(1, min(args.steps, 3)))
    _lib.set_screen_audit(True)
    _lib.screen_audit()
    step()
    audit = _lib.screen_audit()
    _lib.set_screen_audit(False)
    clock = clocks.summary()
    value = results["screened"]["s"]
    plain = results.get("plain fp32", {}).get("s")
    line = {
        "metric": f"{n:,} x {d} {spec['label']} tree time (s) on 1 B200, exact",
        "value": value, "unit": "s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(value * 1e3, 2),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(args.workload, n, d),
        "setup": {"l2": "flushed before every step (256 MB write)", "parallelism": "replicas x1"},
        "e2e": {"value": round(e2e, 4), "unit": "s", "h2d_bytes_per_step": int(X.nbytes),
                "d2h_bytes_per_step": int((n - 1) * 4 * 8)},
        "gpu_launches": int(launches or 0),
        "variants": results,
        "plain_fp32": {"value": plain, "speedup_screened": None if plain is None else
                       round(plain / value, 2)},
        "parity": {"identical_to_plain": results.get("plain fp32", {}).get(
            "identical_to_screened"), "e2e_identical": bool(np.array_equal(tree, screened_tree))},
        "screen_audit": audit_summary(audit),
        "roofline": roofline(kt, d, fp32_peak_tflops(torch), clock),
        "passes": passes_summary(kt, sc),
        "clocks": clock,
    }
    if not args.no_cpu_baseline:
        sample = min(n, args.cpu_sample if args.workload != "c1" else n)
        small = np.ascontiguousarray(X[:sample])
        small_dev = torch.from_numpy(small).cuda()
        small_tree = np.empty((sample - 1) * 4, np.float64)

        def small_step():
            _lib.check(_lib.lib.cuhc_linkage_device(
                ctypes.c_void_p(small_dev.data_ptr()), sample, d, 0, 2.0, spec["linkage"],
                spec["algorithm"], small_tree.ctypes.data_as(f64p)))
        small_step()
        ours_small = timed(small_step, 3)
        if spec["linkage"] == 3:
            line["cpu_baseline"] = sklearn_ward_baseline(X, min(sample, 20_000), ours_small
                                                         if sample <= 20_000 else None)
        else:
            line["cpu_baseline"] = scipy_single_baseline(X, min(sample, 20_000), ours_small
                                                         if sample <= 20_000 else None)
        if not args.no_parity and args.workload != "c4":
            method = "ward" if spec["linkage"] == 3 else "single"
            algorithm = "rnn" if spec["algorithm"] == 3 else "mst"
            line["parity"].update(reference_checks(X, screened_tree, linkage=(method, algorithm)))
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Our arm: the batched workload

def run_batch(args, local_rank):
    """Batched trees of the mixed workload against one call per instance."""
    import torch  # noqa: PLC0415
    sys.path.insert(0, HERE)
    from cuhc_b200 import _batch, _lib  # noqa: PLC0415,F401
    lib = _lib.lib
    i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
    lib.cuhc_trees_batched_device.restype = ctypes.c_int
    lib.cuhc_trees_batched_device.argtypes = [ctypes.c_void_p, i64p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_float, i32p, f64p, f32p]
    inst = make_batch_instances(args.instances)
    groups = []
    for d in (2, 8, 32):
        idx = [i for i, (X, _) in enumerate(inst) if X.shape[1] == d]
        sizes = np.array([len(inst[i][0]) for i in idx], np.int64)
        offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        pts = np.ascontiguousarray(np.concatenate([inst[i][0] for i in idx]))
        ks = np.array([inst[i][1] for i in idx], np.int32)
        trees = np.empty((int(offsets[-1]) - len(idx), 4), np.float64)
        core = np.empty(int(offsets[-1]), np.float32)
        groups.append(dict(d=d, idx=idx, offsets=offsets, pts=pts, dev=torch.from_numpy(pts).cuda(),
                           ks=ks, trees=trees, core=core))

    def device_step():
        for g in groups:
            _lib.check(lib.cuhc_trees_batched_device(
                ctypes.c_void_p(g["dev"].data_ptr()), g["offsets"].ctypes.data_as(i64p),
                len(g["idx"]), g["d"], 0, 2.0, g["ks"].ctypes.data_as(i32p),
                g["trees"].ctypes.data_as(f64p), g["core"].ctypes.data_as(f32p)))

    def host_step():
        for g in groups:
            _lib.check(lib.cuhc_trees_batched(
                g["pts"].ctypes.data_as(f32p), g["offsets"].ctypes.data_as(i64p), len(g["idx"]),
                g["d"], 0, 2.0, g["ks"].ctypes.data_as(i32p), g["trees"].ctypes.data_as(f64p),
                g["core"].ctypes.data_as(f32p)))

    def timed(step, k):
        times = []
        for _ in range(k):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            step()
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        return float(np.mean(times))

    for _ in range(args.warmup):
        device_step()
    launches0 = _lib.launch_count()
    with ClockSampler(local_rank) as clocks:
        t_dev = timed(device_step, args.steps)
    launches = (_lib.launch_count() - launches0) // max(args.steps, 1)
    _lib.set_timing(True)
    _lib.kernel_timing()
    device_step()
    kt = _lib.kernel_timing()
    _lib.set_timing(False)
    t_host = timed(host_step, max(1, min(args.steps, 2)))

    # One call per instance (device-resident points) on every 8th instance.
    sample = list(range(0, len(inst), 8))
    where = {}
    for g in groups:
        for j, i in enumerate(g["idx"]):
            where[i] = (g, j)
    dev = {i: torch.from_numpy(inst[i][0]).cuda() for i in sample}
    trees = {i: np.empty((len(inst[i][0]) - 1, 4), np.float64) for i in sample}
    cores = {i: np.empty(len(inst[i][0]), np.float32) for i in sample}

    def per_instance():
        for i in sample:
            X, k = inst[i]
            if k == 0:
                _lib.check(lib.cuhc_linkage_device(ctypes.c_void_p(dev[i].data_ptr()), len(X),
                                                   X.shape[1], 0, 2.0, 0, 1,
                                                   trees[i].ctypes.data_as(f64p)))
            else:
                _lib.check(lib.cuhc_hdbscan_tree_device(
                    ctypes.c_void_p(dev[i].data_ptr()), len(X), X.shape[1], 0, 2.0, k, 1.0, 0,
                    trees[i].ctypes.data_as(f64p), cores[i].ctypes.data_as(f32p)))

    per_instance()
    t_per = timed(per_instance, 1)
    identical = True
    for i in sample:
        g, j = where[i]
        first = int(g["offsets"][j]) - j
        Z = g["trees"][first:first + len(inst[i][0]) - 1]
        identical &= bool(np.array_equal(Z, trees[i]))
        if inst[i][1]:
            identical &= bool(np.array_equal(g["core"][g["offsets"][j]:g["offsets"][j + 1]],
                                             cores[i]))
    count = len(inst)
    per_rate = len(sample) / t_per
    line = {
        "metric": f"batched exact trees, instances/s on 1 B200 ({count:,} mixed single-linkage / "
                  "HDBSCAN instances, n 64-50k, d 2/8/32)",
        "value": round(count / t_dev, 1), "unit": "instances/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_dev * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": batch_config(count),
        "setup": {"timing": "wall clock around synchronised calls (one call per feature count)",
                  "points": int(sum(len(X) for X, _ in inst))},
        "e2e": {"value": round(count / t_host, 1), "unit": "instances/s",
                "h2d_bytes_per_step": int(sum(g["pts"].nbytes for g in groups)),
                "d2h_bytes_per_step": int(sum(g["trees"].nbytes + g["core"].nbytes
                                              for g in groups))},
        "gpu_launches": int(launches),
        "per_instance": {"value": round(per_rate, 1), "unit": "instances/s",
                         "sample": f"every 8th instance ({len(sample)}), one "
                                   "cuhc_linkage_device / cuhc_hdbscan_tree_device call each",
                         "batched_speedup": round((count / t_dev) / per_rate, 2)},
        "parity": {"identical_to_per_instance_sample": identical},
        "passes": {k: {"ms": round(v[0], 2), "launches": v[1], "tiles": v[2]}
                   for k, v in kt.items()},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def batch_config(count):
    return {"workload": f"{count} instances, seed 4: n log-uniform in [64, 50,000], d in "
                        "{2, 8, 32}, 1-12 blobs + 5% noise; even instances single linkage, "
                        "odd HDBSCAN min_samples 10", "instances": count}


# ---------------------------------------------------------------------------
# Reference arm

def run_reference(args, rank):
    """The reference library on the same data, through its own C ABI (host
    buffers, its default pruning), on rank 0 only."""
    ref = os.path.join(HERE, "oracle", "_ref", "libcuhc.so")
    if rank != 0:
        return None
    if not os.path.exists(ref):
        return {"impl": "reference", "unavailable": "oracle/_ref/libcuhc.so was not built "
                "(the reference sources were absent when build() ran)"}
    L = ctypes.CDLL(ref)
    L.cuhc_hdbscan_tree.argtypes = [f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                    f64p, f32p]
    L.cuhc_linkage.argtypes = [f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                               ctypes.c_int, ctypes.c_int, f64p]
    L.cuhc_set_pruning.argtypes = [ctypes.c_int]
    L.cuhc_set_pruning(0)

    def check(status):
        if status != 0:
            raise RuntimeError(f"reference status {status}")

    if args.workload == "batch":
        inst = make_batch_instances(args.instances)
        sample = list(range(0, len(inst), 8))
        outs = {i: (np.empty((len(inst[i][0]) - 1) * 4, np.float64),
                    np.empty(len(inst[i][0]), np.float32)) for i in sample}

        def step():
            for i in sample:
                X, k = inst[i]
                Z, core = outs[i]
                if k == 0:
                    check(L.cuhc_linkage(X.ctypes.data_as(f32p), len(X), X.shape[1], 0, 2.0, 0,
                                         1, Z.ctypes.data_as(f64p)))
                else:
                    check(L.cuhc_hdbscan_tree(X.ctypes.data_as(f32p), len(X), X.shape[1], 0, 2.0,
                                              k, 1.0, 0, Z.ctypes.data_as(f64p),
                                              core.ctypes.data_as(f32p)))
        config = batch_config(len(inst))
        unit, higher, metric = "instances/s", True, (
            f"batched exact trees, instances/s on 1 B200 ({len(inst):,} mixed single-linkage / "
            "HDBSCAN instances, n 64-50k, d 2/8/32)")
        sample_note = (f"one call per instance on every 8th instance ({len(sample)}); "
                       "the reference has no batched entry point")
    else:
        if args.workload == "hdbscan":
            X = make_blobs_with_noise(n=args.n or N_POINTS)
            tree = np.empty((len(X) - 1, 4), np.float64)
            core = np.empty(len(X), np.float32)

            def step():
                check(L.cuhc_hdbscan_tree(X.ctypes.data_as(f32p), len(X), X.shape[1], 0, 2.0,
                                          MIN_SAMPLES, 1.0, 0, tree.ctypes.data_as(f64p),
                                          core.ctypes.data_as(f32p)))
            metric = METRIC
        else:
            spec = TREES[args.workload]
            X = tree_data(args.workload, args.n)
            tree = np.empty((len(X) - 1, 4), np.float64)

            def step():
                check(L.cuhc_linkage(X.ctypes.data_as(f32p), len(X), X.shape[1], 0, 2.0,
                                     spec["linkage"], spec["algorithm"], tree.ctypes.data_as(f64p)))
            metric = f"{len(X):,} x {X.shape[1]} {spec['label']} tree time (s) on 1 B200, exact"
        config = workload_config(args.workload, *X.shape)
        unit, higher = UNIT, False
        sample_note = "the full workload: the reference library's host code is single-threaded " \
                      "and its passes run on the GPU"

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    seconds = float(np.mean(times))
    value = len(sample) / seconds if args.workload == "batch" else seconds
    value = round(value, 4)
    return {"metric": metric, "value": value, "unit": unit, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(seconds * 1e3, 2), "higher_is_better": higher,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config, "setup": {"pruning": "auto (the reference's default)"},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "cpu_baseline": {"value": value, "unit": unit, "cores": 1, "kind": "reference",
                             "sample": sample_note}}


def main():
    parser = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--workload", choices=["hdbscan", "single32", "c1", "ward", "c4", "batch"],
                        default="hdbscan")
    parser.add_argument("--instances", type=int, default=4096,
                        help="instances of the batch workload")
    parser.add_argument("--no-plain", action="store_true",
                        help="skip the screening-off comparison step")
    parser.add_argument("--no-cpu-baseline", action="store_true",
                        help="skip the CPU baseline and the checkers")
    parser.add_argument("--no-parity", action="store_true",
                        help="skip the checkers (oracle, reference library) of the CPU leg")
    parser.add_argument("--cpu-sample", type=int, default=50_000,
                        help="points of the CPU baseline's sample")
    parser.add_argument("--n", type=int, default=None,
                        help="points of the same recipe (smaller cases for profiling)")
    args = parser.parse_args()

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))

    import torch  # plumbing: device buffers, events, process group  # noqa: PLC0415
    import torch.distributed as dist  # noqa: PLC0415
    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta  # noqa: PLC0415
        dist.init_process_group("nccl", timeout=timedelta(minutes=5))

    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
    elif args.workload == "hdbscan":
        run_hdbscan(args, rank, world, local_rank)
    elif rank == 0 and args.workload == "batch":
        run_batch(args, local_rank)
    elif rank == 0:
        run_tree_workload(args, local_rank)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
