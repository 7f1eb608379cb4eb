"""HDBSCAN extraction (host C++): labels and probabilities identical to
scikit-learn 1.9's tree_to_labels, on stored fixtures (tests/golden/cpu.npz)
and live; plus a hand-built condensed tree with known answers. No GPU."""

import pathlib

import numpy as np
import pytest

from _data import blobs
from cuhc_b200._hdbscan import condense_tree, tree_to_labels
from golden.inputs import CPU_CASES
from oracle import oracle as O

CPU = np.load(pathlib.Path(__file__).resolve().parent / "golden" / "cpu.npz")

try:
    from sklearn.cluster._hdbscan._linkage import HIERARCHY_dtype
    from sklearn.cluster._hdbscan._tree import tree_to_labels as sk_tree_to_labels
except ImportError:  # pragma: no cover
    sk_tree_to_labels = None


@pytest.mark.parametrize("name", [k for k, v in CPU_CASES.items() if v["kind"] == "condense"])
@pytest.mark.parametrize("method", ["eom", "leaf"])
def test_matches_sklearn_fixtures(name, method):
    Z = CPU[f"{name}/tree"]
    for mcs in CPU_CASES[name]["mcs"]:
        key = f"{name}/mcs{mcs}/{method}"
        if f"{key}/labels" not in CPU:
            pytest.skip("fixture made without sklearn")
        labels, probs = tree_to_labels(Z, mcs, method)
        np.testing.assert_array_equal(labels, CPU[f"{key}/labels"])
        np.testing.assert_array_equal(probs, CPU[f"{key}/probabilities"])


def _sk(Z, **params):
    tree = np.empty(len(Z), dtype=HIERARCHY_dtype)
    tree["left_node"], tree["right_node"] = Z[:, 0], Z[:, 1]
    tree["value"], tree["cluster_size"] = Z[:, 2], Z[:, 3]
    try:
        return sk_tree_to_labels(tree, **params)
    except TypeError as error:  # sklearn's epsilon climb on NumPy >= 2.5
        pytest.skip(str(error))


@pytest.mark.skipif(sk_tree_to_labels is None, reason="sklearn private API missing")
@pytest.mark.parametrize("params", [
    {}, {"cluster_selection_method": "leaf"}, {"cluster_selection_epsilon": 0.5},
    {"cluster_selection_method": "leaf", "cluster_selection_epsilon": 0.5},
    {"allow_single_cluster": True, "min_cluster_size": 100}, {"max_cluster_size": 60},
    {"allow_single_cluster": True, "cluster_selection_epsilon": 2.0},
], ids=lambda p: ",".join(f"{k}={v}" for k, v in p.items()) or "default")
@pytest.mark.parametrize("k", [1, 5, 15])
def test_matches_sklearn_live(params, k):
    params = {"min_cluster_size": 10, **params}
    Z, _ = O.hdbscan_tree(blobs(800, 3, centers=5, noise=0.15, seed=k), k)
    ref_labels, ref_probs = _sk(Z, **params)
    mcs = params.pop("min_cluster_size")
    labels, probs = tree_to_labels(Z, mcs, **params)
    np.testing.assert_array_equal(labels, ref_labels)
    np.testing.assert_array_equal(probs, ref_probs)


def test_condense_matches_oracle():
    Z, _ = O.hdbscan_tree(blobs(2000, 4, noise=0.1, seed=3), 5)
    for mcs in (2, 5, 25):
        for ours, ref in zip(condense_tree(Z, mcs), O.condense_tree(Z, mcs)):
            np.testing.assert_array_equal(ours, ref)


def small_condensed_tree():
    """Ten points: root 10 splits at distance 3 into 11 (points 0-5) and 12
    (points 6-9); 11 splits at distance 0.4 into 13 (0-2) and 14 (3-5);
    points leave their leaf at distance 0.2."""
    rows = [(10, 11, 1 / 3.0, 6), (10, 12, 1 / 3.0, 4), (11, 13, 1 / 0.4, 3),
            (11, 14, 1 / 0.4, 3)]
    rows += [(13, p, 5.0, 1) for p in range(3)] + [(14, p, 5.0, 1) for p in range(3, 6)]
    rows += [(12, p, 5.0, 1) for p in range(6, 10)]
    return rows


def tree_from_condensed(rows, n=10):
    """A single-linkage tree whose condensed tree (min_cluster_size 3) is
    `rows`: points join their leaf at 0.2, leaves join at the split heights."""
    Z, next_id, members = [], n, {}

    def join(a, b, h):
        nonlocal next_id
        size = members.get(a, 1) + members.get(b, 1)
        Z.append([min(a, b), max(a, b), h, size])
        members[next_id] = size
        next_id += 1
        return next_id - 1

    def chain(points):
        node = points[0]
        for p in points[1:]:
            node = join(node, p, 0.2)
        return node

    c13, c14, c12 = chain([0, 1, 2]), chain([3, 4, 5]), chain([6, 7, 8, 9])
    c11 = join(c13, c14, 0.4)
    join(c11, c12, 3.0)
    Z = np.array(Z, dtype=np.float64)
    return Z[np.argsort(Z[:, 2], kind="stable")] if False else Z


@pytest.mark.parametrize("epsilon, allow_single, expected", [
    (0.0, False, [{0, 1, 2}, {3, 4, 5}, {6, 7, 8, 9}]),
    (0.3, False, [{0, 1, 2}, {3, 4, 5}, {6, 7, 8, 9}]),
    (0.5, False, [{0, 1, 2, 3, 4, 5}, {6, 7, 8, 9}]),
    (5.0, False, [{0, 1, 2, 3, 4, 5}, {6, 7, 8, 9}]),
    (5.0, True, [set(range(10))]),
])
def test_leaf_selection_with_epsilon_known_answers(epsilon, allow_single, expected):
    """Known answers of the leaf method with an epsilon (the reference's
    tests/test_hdbscan.py:245-285 case, restated on a tree built here)."""
    Z = tree_from_condensed(small_condensed_tree())
    labels, _ = tree_to_labels(Z, 3, "leaf", allow_single, epsilon)
    groups = {frozenset(np.flatnonzero(labels == lab).tolist()) for lab in set(labels.tolist())}
    assert (labels >= 0).all()
    assert groups == {frozenset(g) for g in expected}


def test_pure_noise_labels():
    Z, _ = O.hdbscan_tree(np.random.default_rng(5).uniform(size=(200, 2)).astype(np.float32), 50)
    labels, probs = tree_to_labels(Z, 50)
    if sk_tree_to_labels is not None:
        ref_labels, ref_probs = _sk(Z, min_cluster_size=50)
        np.testing.assert_array_equal(labels, ref_labels)
        np.testing.assert_array_equal(probs, ref_probs)
