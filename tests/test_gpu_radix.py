"""GPU: core distances by radix select (any k) equal the per-row list path
bit for bit where both run (k <= 256), and the oracle beyond; the trees
built on them equal the oracle's (reference test_hdbscan.py:162-179 pins
fused == radix)."""

import numpy as np
import pytest

from _data import blobs, normal
from cuhc_b200._hdbscan import hdbscan_tree
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [1, 7, 25, 64, 200])
@pytest.mark.parametrize("metric", ["euclidean", "manhattan", "cosine"])
def test_radix_equals_lists(k, metric):
    X = blobs(1500, 6, noise=0.1, seed=k)
    Z1, c1 = hdbscan_tree(X, k, metric=metric, core_method="radix")
    Z2, c2 = hdbscan_tree(X, k, metric=metric, core_method="auto")
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(Z1, Z2)


@pytest.mark.parametrize("k", [257, 300, 1000, 1200])
def test_large_k_matches_oracle(k):
    X = blobs(1200, 4, noise=0.1, seed=k)
    Z, core = hdbscan_tree(X, k)
    Z_ref, core_ref = O.hdbscan_tree(X, k)
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Z, Z_ref)


def test_chunked_rows_match_oracle():
    # 20,000 points: the 512 MiB distance block holds 52 row tiles, so the
    # 157 row tiles run in four chunks.
    X = normal(20000, 8, seed=11)
    _, core = hdbscan_tree(X, 300, core_method="radix")
    rows = (0, 400)
    np.testing.assert_array_equal(core[:400], O.core_distances(X, 300, rows=rows))
    idx = np.arange(19600, 20000)
    np.testing.assert_array_equal(core[idx], O.core_distances(X, 300, rows=(19600, 20000)))


def test_duplicates_give_zero_core():
    X = np.repeat(normal(40, 3, seed=2), 300, axis=0)
    _, core = hdbscan_tree(X, 290, core_method="radix")
    np.testing.assert_array_equal(core, np.zeros(len(X), np.float32))
