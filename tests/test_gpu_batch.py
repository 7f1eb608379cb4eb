"""GPU: batched trees (cuhc_trees_batched) are bit-identical to the
per-instance calls, for mixed sizes (tile edges, tiny instances),
single-linkage and HDBSCAN instances in one batch, several feature counts,
duplicates, and a metric without the tensor-core screen."""

import numpy as np
import pytest

import cuhc_b200 as C
from _data import blobs, normal
from cuhc_b200._hdbscan import hdbscan_tree

pytestmark = pytest.mark.gpu


def _per_instance(X, k, metric="euclidean"):
    if k == 0:
        return C.linkage(X, "single", metric=metric), np.zeros(len(X), np.float32)
    return hdbscan_tree(X, k, metric=metric)


def _check(instances, ks, metric="euclidean"):
    got = C.batched_trees(instances, ks, metric=metric)
    for X, k, (Z, core) in zip(instances, ks, got):
        Z_ref, core_ref = _per_instance(X, k, metric)
        np.testing.assert_array_equal(core, core_ref)
        np.testing.assert_array_equal(Z, Z_ref)


SIZES = [1, 2, 3, 10, 64, 127, 128, 129, 255, 256, 257, 500, 1000, 2500, 4000]


@pytest.mark.parametrize("d", [2, 8, 32])
def test_mixed_batch(d):
    rng = np.random.default_rng(d)
    instances, ks = [], []
    for i, n in enumerate(SIZES):
        instances.append(blobs(n, d, noise=0.05, seed=100 * d + i) if n >= 10 else normal(n, d, seed=i))
        ks.append(0 if i % 2 == 0 else int(min(n, rng.choice([1, 5, 10, 25]))))
    _check(instances, ks)


def test_duplicates_and_grids():
    cube = np.indices((8, 8, 8)).reshape(3, -1).T.astype(np.float32)  # integer grid: ties
    instances = [np.repeat(normal(50, 3, seed=1), 4, axis=0), np.zeros((300, 3), np.float32),
                 blobs(700, 3, seed=3), cube]
    _check(instances, [0, 6, 10, 0])


def test_plain_metric():
    instances = [blobs(n, 5, seed=n) for n in (40, 300, 1200)]
    _check(instances, [0, 7, 3], metric="manhattan")


def test_repeat_is_identical():
    instances = [blobs(n, 8, noise=0.1, seed=n) for n in (200, 900, 3000)]
    a = C.batched_trees(instances, [10, 0, 10])
    b = C.batched_trees(instances, [10, 0, 10])
    for (Za, ca), (Zb, cb) in zip(a, b):
        np.testing.assert_array_equal(Za, Zb)
        np.testing.assert_array_equal(ca, cb)


def test_cosine_batch():
    """Cosine, which runs on the tensor-core screen: every batched tree equals
    its own call's (zero points and antiparallel copies included)."""
    instances = []
    for n in (3, 129, 700, 2000):
        X = blobs(n, 16, noise=0.1, seed=n)
        if n >= 129:
            X[:4] = 0.0
            X[4:20] = -X[20:36]
        instances.append(X)
    _check(instances, [0, 5, 0, 9], metric="cosine")
