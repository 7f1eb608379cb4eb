"""Seeded test data."""

import numpy as np


def blobs(n=400, d=8, centers=5, noise=0.0, seed=0, std=(0.5, 2.0)):
    """Gaussian blobs (float32), optionally with uniform background noise.
    Continuous values, so exactly tied distances are vanishingly rare."""
    rng = np.random.default_rng(seed)
    n_noise = int(n * noise)
    m = n - n_noise
    centres = rng.uniform(-10, 10, (centers, d))
    stds = rng.uniform(std[0], std[1], centers)
    label = rng.integers(0, centers, m)
    X = centres[label] + rng.standard_normal((m, d)) * stds[label, None]
    if n_noise:
        X = np.vstack([X, rng.uniform(X.min(0), X.max(0), (n_noise, d))])
    return X.astype(np.float32)


def normal(n, d, seed=0):
    return np.random.default_rng(seed).standard_normal((n, d)).astype(np.float32)


def grid(side=20):
    """Integer grid: huge numbers of exactly equal distances."""
    g = np.stack(np.meshgrid(np.arange(side), np.arange(side)), axis=-1).reshape(-1, 2)
    return g.astype(np.float32)


def subtree_sizes(children, n):
    sizes = np.ones(2 * n - 1, dtype=np.int64)
    for i, (a, b) in enumerate(np.asarray(children, dtype=np.int64)):
        sizes[n + i] = sizes[a] + sizes[b]
    return sizes[n:]


def tree_clusters(Z):
    """{(smallest point, size): height} for every cluster a merge tree makes:
    the dendrogram independent of the order of tied merges."""
    Z = np.asarray(Z)
    n = len(Z) + 1
    smallest = np.empty(2 * n - 1, dtype=np.int64)
    smallest[:n] = np.arange(n)
    out = {}
    for i, (a, b, h, s) in enumerate(Z):
        smallest[n + i] = min(smallest[int(a)], smallest[int(b)])
        out[(int(smallest[n + i]), int(s))] = float(h)
    return out


def assert_same_dendrogram(Z, ref, rtol=1e-4, atol=1e-5):
    ours, theirs = tree_clusters(Z), tree_clusters(ref)
    assert ours.keys() == theirs.keys(), f"{len(ours.keys() ^ theirs.keys())} clusters differ"
    keys = sorted(theirs)
    np.testing.assert_allclose([ours[k] for k in keys], [theirs[k] for k in keys],
                               rtol=rtol, atol=atol)


def assert_well_formed(Z, n):
    ids = np.asarray(Z)[:, :2].astype(np.int64)
    assert Z.shape == (n - 1, 4)
    assert np.all(ids[:, 0] < ids[:, 1])
    np.testing.assert_array_equal(np.sort(ids.ravel()), np.arange(2 * n - 2))
    assert np.all(ids < n + np.arange(n - 1)[:, None])
    np.testing.assert_array_equal(Z[:, 3], subtree_sizes(ids, n))


def assert_same_partition(ours, ref):
    ours, ref = np.asarray(ours), np.asarray(ref)
    assert ours.shape == ref.shape
    np.testing.assert_array_equal(ours == -1, ref == -1)
    keep = ref != -1
    pairs = set(zip(ours[keep].tolist(), ref[keep].tolist()))
    assert len(pairs) == len({a for a, _ in pairs}) == len({b for _, b in pairs})
