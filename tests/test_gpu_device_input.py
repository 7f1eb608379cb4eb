"""GPU: arrays already in GPU memory go to the device entry points.

PyTorch CUDA tensors (through __cuda_array_interface__) and DLPack
capsule producers are read in place by linkage, hdbscan_tree, HDBSCAN,
AgglomerativeClustering and pairwise_distances; results equal the host
path's bit for bit. The reference plans this input path
(docs/architecture.md:380-381)."""

import numpy as np
import pytest

import cuhc_b200 as C
from _data import blobs
from cuhc_b200._hdbscan import hdbscan_tree

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


class DLPackOnly:
    """An array exposing only the DLPack protocol (no CUDA array interface)."""

    def __init__(self, tensor):
        self.tensor = tensor

    def __dlpack__(self, stream=None):
        return self.tensor.__dlpack__()

    def __dlpack_device__(self):
        return self.tensor.__dlpack_device__()


def test_linkage_and_hdbscan_from_device_arrays():
    X = blobs(3000, 8, noise=0.1, seed=61)
    dev = torch.from_numpy(X).cuda()
    np.testing.assert_array_equal(C.linkage(dev, "single"), C.linkage(X, "single"))
    np.testing.assert_array_equal(C.linkage(DLPackOnly(dev), "single"), C.linkage(X, "single"))
    np.testing.assert_array_equal(C.linkage(dev[:1500], "ward"), C.linkage(X[:1500], "ward"))
    for a, b in zip(hdbscan_tree(dev, 10), hdbscan_tree(X, 10)):
        np.testing.assert_array_equal(a, b)
    labels = C.HDBSCAN(min_cluster_size=15).fit(dev).labels_
    np.testing.assert_array_equal(labels, C.HDBSCAN(min_cluster_size=15).fit(X).labels_)
    agg = C.AgglomerativeClustering(n_clusters=4, linkage="single").fit(dev)
    np.testing.assert_array_equal(agg.labels_, C.AgglomerativeClustering(
        n_clusters=4, linkage="single").fit(X).labels_)


def test_pairwise_distances_on_device():
    X, Y = blobs(700, 6, seed=62), blobs(300, 6, seed=63)
    out = C.pairwise_distances(torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda(),
                               metric="manhattan")
    assert out.is_cuda and out.shape == (700, 300)
    np.testing.assert_array_equal(out.cpu().numpy(), C.pairwise_distances(X, Y, "manhattan"))


def test_device_arrays_are_validated():
    with pytest.raises(ValueError, match="float32"):
        C.linkage(torch.zeros((10, 3), dtype=torch.float64, device="cuda"), "single")
    with pytest.raises(ValueError, match="C-contiguous"):
        C.linkage(torch.zeros((3, 10), device="cuda").t(), "single")
