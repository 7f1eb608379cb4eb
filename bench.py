#!/usr/bin/env python
"""Benchmark of the exact HDBSCAN tree (1,000,000 x 8, min_samples 25).

Workload: 20 isotropic Gaussian blobs (centres uniform in [-10, 10]^8,
std 1.0, 45,000 points each) plus 100,000 points uniform over their bounding
box, float32, shuffled, seed 1 -- synthetic data of the headline shape. One
step = one full exact HDBSCAN single-linkage tree: core distances (k = 25),
Borůvka MST of mutual reachability, sorted merges, scipy-format Z and the
core distances copied to the host.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). `value` is the device-resident time per tree
(points already in HBM, cuhc_hdbscan_tree_device); `e2e` is the same through
the host API (cuhc_hdbscan_tree) with pinned host buffers, copies included.
`--impl reference` runs the reference library (shangar21/cuhc built from its
sources for sm_100a, oracle/_ref/libcuhc.so) through its own C ABI with host
buffers and its default pruning, on the same data and GPU. With N > 1 GPUs
each rank builds its own tree (replicas; the path does not shard).
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

METRIC = "1M-pt single/HDBSCAN MST time (s) on 1 B200, screened vs plain FP32, exact tree"
UNIT = "s"
N_POINTS, N_FEATURES, MIN_SAMPLES = 1_000_000, 8, 25
L2_FLUSH_BYTES = 256 << 20
HERE = os.path.dirname(os.path.abspath(__file__))


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


def run_batch(args, local_rank):
    """Batched trees of the mixed workload against one call per instance."""
    import torch  # noqa: PLC0415
    sys.path.insert(0, HERE)
    from cuhc_b200 import _batch, _lib  # noqa: PLC0415,F401
    lib = _lib.lib
    i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
    f32, f64 = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
    lib.cuhc_trees_batched_device.restype = ctypes.c_int
    lib.cuhc_trees_batched_device.argtypes = [ctypes.c_void_p, i64p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_float, i32p, f64, f32]
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
                g["trees"].ctypes.data_as(f64), g["core"].ctypes.data_as(f32)))

    def host_step():
        for g in groups:
            _lib.check(lib.cuhc_trees_batched(
                g["pts"].ctypes.data_as(f32), g["offsets"].ctypes.data_as(i64p), len(g["idx"]),
                g["d"], 0, 2.0, g["ks"].ctypes.data_as(i32p), g["trees"].ctypes.data_as(f64),
                g["core"].ctypes.data_as(f32)))

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
    with ClockSampler(local_rank) as clocks:
        t_dev = timed(device_step, args.steps)
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
                                                   trees[i].ctypes.data_as(f64)))
            else:
                _lib.check(lib.cuhc_hdbscan_tree_device(
                    ctypes.c_void_p(dev[i].data_ptr()), len(X), X.shape[1], 0, 2.0, k, 1.0, 0,
                    trees[i].ctypes.data_as(f64), cores[i].ctypes.data_as(f32)))

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
        "config": {"workload": f"{count} instances, seed 4: n log-uniform in [64, 50,000], d in "
                               "{2, 8, 32}, 1-12 blobs + 5% noise; even instances single "
                               "linkage, odd HDBSCAN min_samples 10",
                   "points": int(sum(len(X) for X, _ in inst)),
                   "timing": "wall clock around synchronised calls (one call per feature count)"},
        "e2e": {"value": round(count / t_host, 1), "unit": "instances/s",
                "h2d_bytes_per_step": int(sum(g["pts"].nbytes for g in groups)),
                "d2h_bytes_per_step": int(sum(g["trees"].nbytes + g["core"].nbytes
                                              for g in groups))},
        "per_instance": {"value": round(per_rate, 1), "unit": "instances/s",
                         "sample": f"every 8th instance ({len(sample)}), one "
                                   "cuhc_linkage_device / cuhc_hdbscan_tree_device call each",
                         "batched_speedup": round((count / t_dev) / per_rate, 2)},
        "identical_sample": identical,
        "passes": {k: {"ms": round(v[0], 2), "launches": v[1], "tiles": v[2]}
                   for k, v in kt.items()},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def run_tree_workload(args, local_rank):
    """Single-linkage 4M x 16 (radius proposal off / on) or Ward 1M x 32 (RNN
    rounds): device-resident time per tree through the C ABI."""
    import torch  # noqa: PLC0415
    sys.path.insert(0, HERE)
    import cuhc_b200 as C  # noqa: PLC0415
    from cuhc_b200 import _lib  # noqa: PLC0415
    from cuhc_b200.train_radius import make_anisotropic_blobs  # noqa: PLC0415
    lib = _lib.lib
    if args.workload == "c4":
        X = make_anisotropic_blobs(3, args.n or 4_000_000)
        linkage_id, algorithm, label = 0, 1, "single linkage (Borůvka)"
    else:
        X = np.random.default_rng(2).standard_normal((args.n or 1_000_000, 32)).astype(np.float32)
        linkage_id, algorithm, label = 3, 3, "Ward (RNN rounds)"
    n, d = X.shape
    dev = torch.from_numpy(X).cuda()
    tree = np.empty((n - 1) * 4, np.float64)

    def step():
        _lib.check(lib.cuhc_linkage_device(ctypes.c_void_p(dev.data_ptr()), n, d, 0, 2.0,
                                           linkage_id, algorithm,
                                           tree.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def timed(k):
        times = []
        for _ in range(k):
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            step()
            e.record()
            e.synchronize()
            times.append(s.elapsed_time(e) / 1e3)
        return float(np.mean(times))

    results = {}
    variants = [("screened", "auto", None)]
    if args.workload == "c4":
        variants.append(("screened + radius proposal", "auto", "model"))
    variants.append(("plain fp32", "off", None))
    reference_tree = None
    with ClockSampler(local_rank) as clocks:
        for name, screen, radius in variants:
            _lib.set_screen(screen)
            if radius:
                meta = C.load_radius_model()
            for _ in range(args.warmup):
                step()
            C.radius_stats()
            t = timed(args.steps)
            stats = C.radius_stats()
            results[name] = {"s": round(t, 4)}
            if radius:
                results[name]["certified_share"] = round(
                    stats["certified"] / max(1, stats["proposed"]), 4)
                results[name]["model"] = f"trained on seeds {list(meta['seeds'])}, " \
                                         f"n = {int(meta['n'])}, {int(meta['rows'])} rows"
                C.set_radius_model(None)
            if reference_tree is None:
                reference_tree = tree.copy()
            results[name]["identical_tree"] = bool(np.array_equal(tree, reference_tree))
    _lib.set_screen("auto")
    best = min(v["s"] for v in results.values())
    line = {
        "metric": f"{n:,} x {d} {label} tree time (s) on 1 B200, exact",
        "value": results["screened"]["s"], "unit": "s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(results["screened"]["s"] * 1e3, 1),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": ("4M x 16: 50 Gaussian clusters (shared random covariance, "
                                "eigenvalues log-uniform in [0.05, 5]) + 5% noise, seed 3")
                   if args.workload == "c4" else "1M x 32 standard normal, seed 2",
                   "n": n, "d": d, "best_s": best},
        "variants": results,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


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


def cpu_baseline(X):
    """The CPU oracle (C restatement, OpenMP on every host core) timed on a
    bounded sample: core distances of 6,000 rows against all points. A full
    tree evaluates ~1.5 n^2 pairs (n^2 for the core distances, n^2 / 2 for
    Prim's MST), so the sample's time per pair scales to the full workload."""
    sys.path.insert(0, HERE)
    from oracle import oracle as O  # noqa: PLC0415
    rows = 6000
    O.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    O.core_distances(X, MIN_SAMPLES, rows=(0, rows))
    elapsed = time.perf_counter() - t0
    per_pair = elapsed / (rows * len(X))
    full = 1.5 * len(X) ** 2 * per_pair
    return {"value": round(full, 1), "unit": UNIT, "cores": O.threads(), "kind": "port",
            "sample": f"core distances of {rows} rows x {len(X)} points in {elapsed:.1f} s, "
                      f"scaled by 1.5 n^2 pairs per tree"}


def run_reference(args, rank, world):
    """The reference library on the same data, through its own C ABI."""
    ref = os.path.join(HERE, "oracle", "_ref", "libcuhc.so")
    config = {"workload": "hdbscan 1,000,000 x 8, 20 blobs + 10% noise, min_samples 25",
              "n": N_POINTS, "d": N_FEATURES, "min_samples": MIN_SAMPLES, "pruning": "auto"}
    if rank != 0:
        return None
    if not os.path.exists(ref):
        return {"impl": "reference", "unavailable": "oracle/_ref/libcuhc.so was not built "
                "(the reference sources were absent when build() ran)"}
    L = ctypes.CDLL(ref)
    f32, f64 = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
    L.cuhc_hdbscan_tree.argtypes = [f32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                    ctypes.c_int, ctypes.c_float, ctypes.c_int, f64, f32]
    L.cuhc_set_pruning.argtypes = [ctypes.c_int]
    X = make_blobs_with_noise()
    tree = np.empty((len(X) - 1, 4), np.float64)
    core = np.empty(len(X), np.float32)
    L.cuhc_set_pruning(0)

    def step():
        status = L.cuhc_hdbscan_tree(X.ctypes.data_as(f32), len(X), X.shape[1], 0, 2.0,
                                     MIN_SAMPLES, 1.0, 0, tree.ctypes.data_as(f64),
                                     core.ctypes.data_as(f32))
        if status != 0:
            raise RuntimeError(f"reference status {status}")

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    value = float(np.mean(times))
    return {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(value * 1e3, 2), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": 1,
                             "kind": "reference",
                             "sample": "the full workload: the reference library's host code "
                                       "is single-threaded and its passes run on the GPU"}}


def main():
    parser = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--workload", choices=["hdbscan", "batch", "c4", "ward"],
                        default="hdbscan",
                        help="hdbscan: the headline tree; batch: many small instances; c4: "
                             "4M x 16 single linkage; ward: 1M x 32 Ward")
    parser.add_argument("--instances", type=int, default=4096,
                        help="instances of the batch workload")
    parser.add_argument("--no-plain", action="store_true",
                        help="skip the screening-off comparison step")
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

    if args.workload in ("c4", "ward"):
        if rank == 0 and args.impl == "ours":
            run_tree_workload(args, local_rank)
        elif rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the secondary workloads are "
                              "measured against the reference in the headline arm only"}),
                  flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    if args.workload == "batch":
        if rank == 0 and args.impl == "ours":
            run_batch(args, local_rank)
        elif rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched "
                              "entry point; its per-instance calls are the batch line's "
                              "per_instance figure"}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    sys.path.insert(0, HERE)
    from cuhc_b200 import _lib  # noqa: PLC0415

    X = make_blobs_with_noise(n=args.n or N_POINTS)
    n, d = X.shape
    f32, f64 = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
    X_dev = torch.from_numpy(X).cuda()
    X_pin = torch.from_numpy(X).pin_memory()
    tree_pin = torch.empty((n - 1) * 4, dtype=torch.float64).pin_memory()
    core_pin = torch.empty(n, dtype=torch.float32).pin_memory()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    tree_ptr = ctypes.cast(tree_pin.data_ptr(), f64)
    core_ptr = ctypes.cast(core_pin.data_ptr(), f32)

    def device_step():
        _lib.check(_lib.lib.cuhc_hdbscan_tree_device(
            ctypes.c_void_p(X_dev.data_ptr()), n, d, 0, 2.0, MIN_SAMPLES, 1.0, 0, tree_ptr,
            core_ptr))

    def host_step():
        _lib.check(_lib.lib.cuhc_hdbscan_tree(
            ctypes.cast(X_pin.data_ptr(), f32), n, d, 0, 2.0, MIN_SAMPLES, 1.0, 0, tree_ptr,
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

    # Kernel-level figures: the pass kernels timed on their own stream.
    _lib.set_timing(True)
    _lib.kernel_timing()
    _lib.screen_counters()
    timed(device_step, 1)
    kt = _lib.kernel_timing()
    sc = _lib.screen_counters()
    _lib.set_timing(False)

    # The same step with tensor-core screening switched off (plain FP32 passes).
    plain = float("nan")
    if not args.no_plain:
        _lib.set_screen("off")
        device_step()
        plain = float(np.mean(timed(device_step, max(1, min(args.steps, 3)))))
        _lib.set_screen("auto")

    # End to end through the host API (pinned buffers, copies included).
    for _ in range(1):
        host_step()
    e2e_times = timed(host_step, args.steps)
    e2e = float(np.mean(e2e_times))

    # Max over ranks.
    t = torch.tensor([per_step, e2e, plain], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    per_step, e2e, plain = float(t[0]), float(t[1]), float(t[2])

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        fp32 = fp32_peak_tflops(torch)
        # Dominant kernel: the pass kind with the most device time.
        kind, (ms, nl, tiles) = max(kt.items(), key=lambda kv: kv[1][0])
        screened = kind.startswith("screen")
        pairs = tiles * 128 * 128
        sgemm = f"cuBLAS SGEMM 8192^3 with TF32 off, measured in this run: {fp32:.2f} TFLOP/s"
        if screened:
            # Screened pass: 2d tensor FLOP per evaluated pair (the -2 X Y^T
            # product) against the TF32 rate, half the measured bf16 burst.
            peak = peaks["bf16_tflops"] / 2 if peaks.get("bf16_tflops") else None
            achieved = pairs * 2 * d / (ms / 1e3) / 1e12 if ms > 0 else 0.0
            k_pad = (3 * d + 4 + 7) // 8 * 8
            issued = pairs * 2 * k_pad / (ms / 1e3) / 1e12 if ms > 0 else 0.0
            roof = {"bound": "tensor", "kernel": kind, "achieved": round(achieved, 2),
                    "peak": round(peak, 1) if peak else None, "unit": "TFLOP/s",
                    "frac": round(achieved / peak, 4) if peak else None, "traffic": None,
                    "peak_source": f"TF32 = half the bf16 burst {peaks.get('bf16_tflops')} "
                                   f"TFLOP/s ({peak_kind})",
                    "work": f"{tiles} tiles x 16384 pairs x 2d FLOP in {nl} launches, "
                            f"{ms:.1f} ms",
                    "issued_tflops": round(issued, 2),
                    "fp32_equivalent": {"achieved": round(pairs * 3 * d / (ms / 1e3) / 1e12, 2),
                                        "peak": round(fp32, 2), "peak_source": sgemm}}
        else:
            # Plain pass: 3d FP32 FLOP per evaluated pair (d subtractions + d
            # fused multiply-adds) against the FP32 pipe.
            achieved = pairs * 3 * d / (ms / 1e3) / 1e12 if ms > 0 else 0.0
            roof = {"bound": "fp32", "kernel": kind, "achieved": round(achieved, 2),
                    "peak": round(fp32, 2), "unit": "TFLOP/s",
                    "frac": round(achieved / fp32, 3) if fp32 else None, "traffic": None,
                    "peak_source": sgemm,
                    "work": f"{tiles} tiles x 16384 pairs x 3d FLOP in {nl} launches, "
                            f"{ms:.1f} ms"}
        line = {
            "metric": METRIC, "value": round(per_step, 4), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 2),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"hdbscan {n:,} x 8, 20 blobs + 10% noise, min_samples 25",
                       "n": n, "d": d, "min_samples": MIN_SAMPLES,
                       "path": "tcgen05 TF32 screen + exact FP32 recheck" if screened
                               else "plain exact fp32",
                       "l2": "flushed before every step (256 MB write)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(e2e, 4), "unit": UNIT, "h2d_bytes_per_step": int(X.nbytes),
                    "d2h_bytes_per_step": int((n - 1) * 4 * 8 + n * 4)},
            "gpu_launches": int(launches),
            "roofline": roof,
            "plain_fp32": {"value": None if np.isnan(plain) else round(plain, 4), "unit": UNIT,
                           "note": "same step with tensor-core screening off"},
            "passes": {**{k: {"ms": round(v[0], 2), "launches": v[1], "tiles": v[2]}
                          for k, v in kt.items()},
                       "screen": {**sc, "rechecks_per_pair": round(
                           sc["rechecks"] / max(1, 16384 * sum(
                               v[2] for k, v in kt.items() if k.startswith("screen"))), 6)},
                       "tiles_per_step": int((stats1[0] - stats0[0]) / max(args.steps, 1)),
                       "rounds_per_step": (stats1[3] - stats0[3]) / max(args.steps, 1)},
            "clocks": clocks.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(X)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
