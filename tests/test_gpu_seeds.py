"""GPU: HDBSCAN's Borůvka rounds seeded from the k-NN lists.

The core-distance pass keeps every point's k-NN list; each round then seeds
a row with its lightest list edge to another component and settles the row
outright when that edge weighs the row's core distance and no point outside
the list ties the k-th distance. These cases put ties at the k-th distance
everywhere (integer grids, duplicated points, one-ulp rings), where a wrong
tie flag or a wrong settle would change which of several equal-weight edges
a row reports; every tree must equal the CPU oracle's bit for bit, screened
or plain, pruned or not.
"""

import numpy as np
import pytest

from _data import blobs, grid
from cuhc_b200 import _lib
from cuhc_b200._hdbscan import hdbscan_tree
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[("on", "always"), ("off", "always"), ("on", "never")],
                ids=["screened", "plain", "screened-unpruned"])
def mode(request):
    screen, prune = request.param
    _lib.set_screen(screen)
    _lib.set_pruning(prune)
    yield
    _lib.set_screen("auto")
    _lib.set_pruning("auto")


def check(X, k):
    Z, core = hdbscan_tree(X, k)
    Z_ref, core_ref = O.hdbscan_tree(X, k)
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Z, Z_ref)


@pytest.mark.parametrize("k", [2, 4, 5, 9, 16, 25])
def test_integer_grid(mode, k):
    check(grid(30), k)


def test_cube_grid_with_duplicates(mode):
    g = np.stack(np.meshgrid(*[np.arange(11)] * 3), axis=-1).reshape(-1, 3).astype(np.float32)
    X = np.ascontiguousarray(np.vstack([g, g[::7]]))
    for k in (3, 7, 8):
        check(X, k)


def test_duplicated_blobs(mode):
    X = np.repeat(blobs(300, 5, centers=4, seed=12), 3, axis=0)
    for k in (2, 3, 4, 10):
        check(X, k)


def test_one_ulp_rings(mode):
    rng = np.random.default_rng(5)
    centres = rng.uniform(-50, 50, (40, 4)).astype(np.float32)
    pts = [centres]
    for c in centres:
        u = rng.standard_normal((12, 4))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        r = np.float32(1.5)
        radii = np.array([r, np.nextafter(r, np.float32(2)), np.nextafter(r, np.float32(1))],
                         np.float32)[rng.integers(0, 3, 12)]
        pts.append((c + u * radii[:, None]).astype(np.float32))
    X = np.ascontiguousarray(np.vstack(pts))
    for k in (5, 10, 13):
        check(X, k)


def test_blobs_with_noise_many_rounds(mode):
    X = blobs(6000, 8, centers=12, noise=0.1, seed=31)
    check(X, 25)
