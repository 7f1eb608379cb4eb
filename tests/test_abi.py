"""The C ABI without a GPU: the library loads, exports every symbol that
include/cuhc.h declares, validates arguments exactly as the reference does
(capi.cu:138-309), and runs its host-only entry points (condensing)."""

import ctypes
import pathlib
import re

import numpy as np
import pytest

from cuhc_b200 import _lib

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "cuhc.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(cuhc_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_reference_boundary():
    reference_eight = {"cuhc_pairwise_distances", "cuhc_linkage", "cuhc_ward_rnn_with_options",
                       "cuhc_hdbscan_tree", "cuhc_condense_tree", "cuhc_set_pruning",
                       "cuhc_prune_stats", "cuhc_error_string"}
    assert reference_eight <= set(declared_symbols())


@pytest.mark.parametrize("symbol", declared_symbols())
def test_library_exports_declared_symbol(symbol):
    assert hasattr(_lib.lib, symbol)


def test_build_targets_sm100a():
    from cuhc_b200 import build  # noqa: PLC0415
    assert "arch=compute_100a,code=sm_100a" in build.ARCH


f32 = ctypes.POINTER(ctypes.c_float)
f64 = ctypes.POINTER(ctypes.c_double)


def _ptr(a, t):
    return a.ctypes.data_as(t)


@pytest.mark.parametrize("n, d, metric, linkage, algorithm, code", [
    (0, 3, 0, 0, 1, -2),    # empty
    (5, 0, 0, 0, 1, -2),    # no features
    (5, 3, 0, 7, 1, -3),    # linkage id
    (5, 3, 0, 1, 1, -4),    # mst needs single
    (5, 3, 2, 3, 3, -4),    # rnn needs euclidean ward
    (5, 3, 0, 0, 3, -4),    # rnn needs ward
    (5, 3, 9, 0, 1, -1),    # metric id
])
def test_linkage_validation_codes(n, d, metric, linkage, algorithm, code):
    X = np.zeros((max(n, 1), max(d, 1)), np.float32)
    Z = np.zeros((max(n - 1, 1), 4))
    assert _lib.lib.cuhc_linkage(_ptr(X, f32), n, d, metric, 2.0, linkage, algorithm,
                                 _ptr(Z, f64)) == code


def test_single_point_linkage_writes_nothing():
    X = np.zeros((1, 3), np.float32)
    Z = np.full((1, 4), 7.0)
    assert _lib.lib.cuhc_linkage(_ptr(X, f32), 1, 3, 0, 2.0, 0, 1, _ptr(Z, f64)) == 0
    assert np.all(Z == 7.0)


@pytest.mark.parametrize("n, k, method, code", [
    (10, 0, 0, -2), (10, 11, 0, -2), (100, 65, 1, -4), (10, 3, 3, -4), (10, 3, -1, -4)])
def test_hdbscan_validation_codes(n, k, method, code):
    X = np.zeros((n, 2), np.float32)
    Z = np.zeros((n - 1, 4))
    core = np.zeros(n, np.float32)
    assert _lib.lib.cuhc_hdbscan_tree(_ptr(X, f32), n, 2, 0, 2.0, k, 1.0, method, _ptr(Z, f64),
                                      _ptr(core, f32)) == code


def test_pairwise_validation_codes():
    X = np.zeros((3, 2), np.float32)
    out = np.zeros((3, 3), np.float32)
    assert _lib.lib.cuhc_pairwise_distances(_ptr(X, f32), 0, None, 3, 2, 0, 2.0,
                                            _ptr(out, f32)) == -2
    assert _lib.lib.cuhc_pairwise_distances(_ptr(X, f32), 3, None, 3, 2, 6, 2.0,
                                            _ptr(out, f32)) == -1


def test_pruning_modes():
    for mode in ("always", "never", "auto"):
        _lib.set_pruning(mode)
    assert _lib.lib.cuhc_set_pruning(3) == -4
    with pytest.raises(KeyError):
        _lib.set_pruning("sometimes")


def test_error_strings():
    for code, text in [(-1, "metric"), (-2, "positive"), (-3, "linkage"), (-4, "algorithm"),
                       (-5, "no finite distance"), (-6, "overflowed"), (-7, "wait"),
                       (-8, "limit")]:
        assert text in _lib.lib.cuhc_error_string(code).decode()


def test_condense_tree_runs_on_the_host():
    from oracle import oracle as O  # noqa: PLC0415
    from cuhc_b200._hdbscan import condense_tree  # noqa: PLC0415
    from _data import blobs  # noqa: PLC0415
    Z, _ = O.hdbscan_tree(blobs(1000, 3, noise=0.1, seed=3), 5)
    for mcs in (2, 10, 50):
        for ours, ref in zip(condense_tree(Z, mcs), O.condense_tree(Z, mcs)):
            np.testing.assert_array_equal(ours, ref)


def test_condense_tree_reports_capacity():
    from oracle import oracle as O  # noqa: PLC0415
    from _data import blobs  # noqa: PLC0415
    Z, _ = O.hdbscan_tree(blobs(300, 3, seed=5), 5)
    i64 = ctypes.POINTER(ctypes.c_int64)
    a = np.zeros(4, np.int64)
    lam = np.zeros(4)
    rows = _lib.lib.cuhc_condense_tree(_ptr(np.ascontiguousarray(Z), f64), 300, 5, 4,
                                       _ptr(a, i64), _ptr(a.copy(), i64), _ptr(lam, f64),
                                       _ptr(a.copy(), i64))
    assert rows < -4


def test_batched_validation_without_gpu():
    """cuhc_trees_batched rejects bad shapes before touching a GPU."""
    import ctypes
    from cuhc_b200 import _batch  # noqa: F401  (declares the argtypes)
    lib = _lib.lib
    pts = np.zeros((10, 2), np.float32)
    tree = np.zeros((10, 4), np.float64)
    core = np.zeros(10, np.float32)

    def call(offsets, ks, count=None, d=2, metric=0):
        off = np.asarray(offsets, np.int64)
        k = np.asarray(ks, np.int32)
        return lib.cuhc_trees_batched(
            pts.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
            off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            len(ks) if count is None else count, d, metric, 2.0,
            k.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            tree.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            core.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))

    assert call([0, 4, 10], [0, 0], count=0) == -2          # no instance
    assert call([1, 4, 10], [0, 0]) == -2                   # offsets[0] != 0
    assert call([0, 4, 4], [0, 0]) == -2                    # empty instance
    assert call([0, 4, 10], [5, 0]) == -2                   # min_samples > rows
    assert call([0, 4, 10], [-1, 0]) == -2
    assert call([0, 4, 10], [0, 1], d=0) == -2
    assert call([0, 4, 10], [0, 1], metric=9) == -1
