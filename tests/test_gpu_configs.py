"""GPU: the measured configurations at their own sizes, bit for bit.

Each test builds the configuration's tree with the tensor-core screen (the
default path the benchmark times) and compares it with
  - the same call with the screen off (the plain exact FP32 passes),
  - the reference library (shangar21/cuhc built from its sources,
    oracle/_ref) with spatial pruning off, its bit-parity mode: ties keep
    original indices there, as here (reference capi.cu:75-77),
  - where the CPU can afford it, the C oracle,
and, for HDBSCAN, the extraction: labels and probabilities against
scikit-learn 1.9's tree_to_labels on the same tree and the condensed tree
against the reference's cuhc_condense_tree (the reference's own contract,
tests/test_hdbscan.py:96-118 and tests/test_spatial_pruning.py:45-73).
"""

import numpy as np
import pytest

import cuhc_b200 as C
from bench import make_batch_instances, make_blobs_with_noise, tree_data
from cuhc_b200 import _lib
from cuhc_b200._hdbscan import condense_tree, hdbscan_tree, tree_to_labels
from oracle import oracle as O

pytestmark = pytest.mark.gpu

needs_reference = pytest.mark.skipif(not O.reference_available(),
                                     reason="reference library (oracle/_ref) not built")


def with_screen(mode, fn):
    _lib.set_screen(mode)
    try:
        return fn()
    finally:
        _lib.set_screen("auto")


@pytest.fixture(scope="module")
def c2():
    """HDBSCAN min_samples 25 on the 1,000,000 x 8 headline recipe."""
    X = make_blobs_with_noise()
    Z, core = with_screen("auto", lambda: hdbscan_tree(X, 25))
    return X, Z, core


def test_c2_screened_equals_plain(c2):
    X, Z, core = c2
    Z_plain, core_plain = with_screen("off", lambda: hdbscan_tree(X, 25))
    np.testing.assert_array_equal(core, core_plain)
    np.testing.assert_array_equal(Z, Z_plain)


@needs_reference
def test_c2_equals_reference(c2):
    X, Z, core = c2
    Z_ref, core_ref = O.reference_hdbscan_tree(X, 25, pruning="never")
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Z, Z_ref)


def test_c2_core_distances_equal_oracle(c2):
    X, _, core = c2
    # The recipe shuffles its points: the first rows are a random sample.
    O.set_threads(0)
    np.testing.assert_array_equal(O.core_distances(X, 25, rows=(0, 3000)), core[:3000])


def test_c2_extraction(c2):
    from sklearn.cluster._hdbscan._linkage import HIERARCHY_dtype  # noqa: PLC0415
    from sklearn.cluster._hdbscan._tree import tree_to_labels as sk_tree_to_labels  # noqa: PLC0415
    _, Z, _ = c2
    labels, probabilities = tree_to_labels(Z, 25)
    tree = np.empty(len(Z), dtype=HIERARCHY_dtype)
    tree["left_node"], tree["right_node"] = Z[:, 0], Z[:, 1]
    tree["value"], tree["cluster_size"] = Z[:, 2], Z[:, 3]
    sk_labels, sk_probabilities = sk_tree_to_labels(tree, min_cluster_size=25)
    np.testing.assert_array_equal(labels, sk_labels)
    np.testing.assert_array_equal(probabilities, sk_probabilities)
    assert len(set(labels.tolist()) - {-1}) >= 20  # the 20 blobs are found


@needs_reference
def test_c2_condensed_tree_equals_reference(c2):
    _, Z, _ = c2
    ours = condense_tree(Z, 25)
    ref = O.reference_condense_tree(Z, 25)
    for a, b in zip(ours, ref):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b))


@pytest.fixture(scope="module")
def single32():
    """Single linkage on 1,000,000 x 32 standard normal."""
    X = tree_data("single32")
    return X, with_screen("auto", lambda: C.linkage(X, "single"))


def test_single32_screened_equals_plain(single32):
    X, Z = single32
    np.testing.assert_array_equal(Z, with_screen("off", lambda: C.linkage(X, "single")))


@needs_reference
def test_single32_equals_reference(single32):
    X, Z = single32
    np.testing.assert_array_equal(Z, O.reference_linkage(X, "single", "mst", pruning="never"))


def test_c3_ward_equals_plain_and_reference():
    """Ward (RNN rounds) on 1,000,000 x 32 standard normal (seed 2)."""
    X = tree_data("ward")
    Z = with_screen("auto", lambda: C.linkage(X, "ward"))
    np.testing.assert_array_equal(Z, with_screen("off", lambda: C.linkage(X, "ward")))
    if O.reference_available():
        np.testing.assert_array_equal(Z, O.reference_linkage(X, "ward", "rnn", pruning="never"))


def test_c4_radius_proposal_never_changes_the_tree():
    """Single linkage on the 4,000,000 x 16 recipe: screened with the learned
    radius proposal equals screened without it; plain equals screened on the
    first 1,000,000 points of the recipe."""
    X = tree_data("c4")
    Z = with_screen("auto", lambda: C.linkage(X, "single"))
    C.load_radius_model()
    try:
        Z_model = with_screen("auto", lambda: C.linkage(X, "single"))
    finally:
        C.set_radius_model(None)
    np.testing.assert_array_equal(Z, Z_model)
    Y = np.ascontiguousarray(X[:1_000_000])
    np.testing.assert_array_equal(with_screen("auto", lambda: C.linkage(Y, "single")),
                                  with_screen("off", lambda: C.linkage(Y, "single")))


def test_c5_every_batched_tree_equals_its_own_call():
    """All 4,096 instances of the batched recipe: every batched tree and core
    vector equals the per-instance call's, and the 64 smallest instances
    equal the oracle's."""
    instances = make_batch_instances()
    out = C.batched_trees([X for X, _ in instances], [k for _, k in instances])
    from cuhc_b200._hdbscan import hdbscan_tree as tree_of  # noqa: PLC0415
    for (X, k), (Z, core) in zip(instances, out):
        if k == 0:
            np.testing.assert_array_equal(Z, C.linkage(X, "single"))
        else:
            Z_one, core_one = tree_of(X, k)
            np.testing.assert_array_equal(Z, Z_one)
            np.testing.assert_array_equal(core, core_one)
    smallest = sorted(range(len(instances)), key=lambda i: len(instances[i][0]))[:64]
    for i in smallest:
        (X, k), (Z, core) = instances[i], out[i]
        if k == 0:
            np.testing.assert_array_equal(Z, O.single_linkage(X))
        else:
            Z_ref, core_ref = O.hdbscan_tree(X, k)
            np.testing.assert_array_equal(core, core_ref)
            np.testing.assert_array_equal(Z, Z_ref)
