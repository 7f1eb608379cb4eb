"""Seeded inputs of the golden fixtures (regenerated, never stored)."""

import numpy as np


def make_input(spec):
    rng = np.random.default_rng(spec["seed"])
    n, d = spec["n"], spec["d"]
    if spec.get("data") == "blobs":
        centres = rng.uniform(-10, 10, (spec.get("centers", 8), d))
        label = rng.integers(0, len(centres), n)
        X = centres[label] + rng.standard_normal((n, d))
        n_noise = int(n * spec.get("noise", 0.0))
        if n_noise:
            X[:n_noise] = rng.uniform(X.min(0), X.max(0), (n_noise, d))
    elif spec.get("data") == "grid":
        side = int(round(n ** 0.5))
        X = np.stack(np.meshgrid(np.arange(side), np.arange(side)), -1).reshape(-1, 2)
    elif spec.get("data") == "duplicates":
        X = np.repeat(rng.standard_normal((n // 4, d)), 4, axis=0)
    else:
        X = rng.standard_normal((n, d))
    return np.ascontiguousarray(X, dtype=np.float32)


# Single-linkage trees vs scipy, condensed trees and sklearn labels.
CPU_CASES = {
    "single_2x3": dict(kind="single", n=2, d=3, seed=1),
    "single_3x2": dict(kind="single", n=3, d=2, seed=2),
    "single_129x8": dict(kind="single", n=129, d=8, seed=3),
    "single_300x32": dict(kind="single", n=300, d=32, seed=4),
    "single_2000x32": dict(kind="single", n=2000, d=32, seed=5),
    "single_1500x8_blobs": dict(kind="single", n=1500, d=8, seed=6, data="blobs"),
    "condense_3000x8": dict(kind="condense", n=3000, d=8, seed=7, data="blobs", noise=0.1,
                            k=5, mcs=(2, 5, 25, 100)),
    "condense_1200x3": dict(kind="condense", n=1200, d=3, seed=8, data="blobs", noise=0.15,
                            k=10, mcs=(10, 40)),
}

# Outputs of the reference library on a GPU (pruning off).
GPU_CASES = {
    "single_2x3": dict(kind="single", n=2, d=3, seed=11),
    "single_127x8": dict(kind="single", n=127, d=8, seed=12),
    "single_128x8": dict(kind="single", n=128, d=8, seed=13),
    "single_129x8": dict(kind="single", n=129, d=8, seed=14),
    "single_5000x32": dict(kind="single", n=5000, d=32, seed=15),
    "single_20000x32": dict(kind="single", n=20000, d=32, seed=0),
    "single_grid": dict(kind="single", n=400, d=2, seed=16, data="grid"),
    "single_dup": dict(kind="single", n=800, d=3, seed=17, data="duplicates"),
    "hdbscan_3000x8": dict(kind="hdbscan", n=3000, d=8, seed=21, data="blobs", noise=0.1, k=25),
    "hdbscan_5000x2": dict(kind="hdbscan", n=5000, d=2, seed=22, data="blobs", noise=0.1, k=5),
    "hdbscan_2000x16_k1": dict(kind="hdbscan", n=2000, d=16, seed=23, data="blobs", k=1),
    "hdbscan_dup_k4": dict(kind="hdbscan", n=800, d=3, seed=24, data="duplicates", k=4),
    "hdbscan_grid_k8": dict(kind="hdbscan", n=400, d=2, seed=25, data="grid", k=8),
    "ward_129x7": dict(kind="ward", n=129, d=7, seed=31, data="blobs"),
    "ward_3000x16": dict(kind="ward", n=3000, d=16, seed=32, data="blobs"),
    "ward_dup": dict(kind="ward", n=400, d=3, seed=33, data="duplicates"),
}
