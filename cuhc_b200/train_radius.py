"""Trains the radius model shipped in cuhc_b200/models/radius_d16.npz.

    python -m cuhc_b200.train_radius [--n 1000000] [--seeds 10-19] [--out PATH]

Data: the 16-feature recipe of `make_anisotropic_blobs` (50 Gaussian clusters,
each with its own random covariance, eigenvalues log-uniform in [0.05, 5],
plus 5% uniform noise) for each seed; every exact single-linkage Borůvka round of
each data set contributes up to 20,000 random rows. Needs a GPU.
"""

import argparse

import numpy as np


def make_anisotropic_blobs(seed, n, d=16, centers=50, noise=0.05):
    """centers clusters of equal weight, centres uniform in [-10, 10]^d, each
    with its own random covariance Q diag(l) Q^T (Q from the QR of a Gaussian
    matrix, l log-uniform in [0.05, 5]), plus `noise` of the points uniform
    over the clusters' bounding box; float32, shuffled."""
    rng = np.random.default_rng(seed)
    n_noise = int(round(n * noise))
    m = n - n_noise
    centres = rng.uniform(-10.0, 10.0, (centers, d))
    transforms = np.empty((centers, d, d))
    for c in range(centers):
        q, _ = np.linalg.qr(rng.standard_normal((d, d)))
        lam = np.exp(rng.uniform(np.log(0.05), np.log(5.0), d))
        transforms[c] = q * np.sqrt(lam)  # x = centre + T z: covariance Q diag(lam) Q^T
    label = np.arange(m) % centers
    z = rng.standard_normal((m, d))
    pts = centres[label] + np.einsum("nij,nj->ni", transforms[label], z)
    lo, hi = pts.min(axis=0), pts.max(axis=0)
    X = np.vstack([pts, rng.uniform(lo, hi, (n_noise, d))]).astype(np.float32)
    return np.ascontiguousarray(X[rng.permutation(n)])


def main():
    from . import _radius  # noqa: PLC0415
    parser = argparse.ArgumentParser()
    parser.add_argument("--n", type=int, default=1_000_000)
    parser.add_argument("--seeds", default="10-19")
    parser.add_argument("--epochs", type=int, default=20)
    parser.add_argument("--out", default=str(_radius.MODEL_PATH))
    args = parser.parse_args()
    a, b = (int(v) for v in args.seeds.split("-"))
    seeds = list(range(a, b + 1))
    data = (make_anisotropic_blobs(s, args.n) for s in seeds)
    params, offset, report = _radius.train_radius_model(data, epochs=args.epochs)
    np.savez(args.out, params=params, offset=np.float32(offset), seeds=np.array(seeds),
             n=np.int64(args.n), rows=np.int64(report["rows"]), losses=report["losses"],
             residual_std=np.float32(report["residual_std"]), quantile=np.float32(0.95))
    print(f"rows {report['rows']}, final loss {report['losses'][-1]:.4f}, "
          f"residual std {report['residual_std']:.4f}, offset {offset:.4f} -> {args.out}")


if __name__ == "__main__":
    main()
