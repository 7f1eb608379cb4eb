"""The allocation-free pairwise-distance entry point.

cuhc_pairwise_distances_noalloc serves callers that cannot allocate GPU
memory (their host framework owns all device memory, or an allocation on
their path could block or fail): inputs and outputs are the caller's device
buffers and the kernel's scratch is a fixed array inside the library. Its
output must equal the regular entry point's, on two calls in a row (the
scratch keeps the previous call's contents, so stale data must not leak into
the second result). This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

from cuhc_b200 import _lib

pytestmark = pytest.mark.gpu

f32 = ctypes.POINTER(ctypes.c_float)
_lib.lib.cuhc_pairwise_distances_noalloc.restype = ctypes.c_int
_lib.lib.cuhc_pairwise_distances_noalloc.argtypes = [
    ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
    ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]


def regular(A, B, metric, p=2.0):
    """The existing host entry point."""
    rows_b = len(A) if B is None else len(B)
    out = np.empty((len(A), rows_b), np.float32)
    _lib.check(_lib.lib.cuhc_pairwise_distances(
        A.ctypes.data_as(f32), len(A), None if B is None else B.ctypes.data_as(f32), rows_b,
        A.shape[1], metric, p, out.ctypes.data_as(f32)))
    return out


def no_alloc(torch, A, B, metric, p=2.0):
    """The new entry point on device buffers the test allocates."""
    dA = torch.from_numpy(A).cuda()
    dB = None if B is None else torch.from_numpy(B).cuda()
    rows_b = len(A) if B is None else len(B)
    out = torch.full((len(A), rows_b), float("nan"), device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib.cuhc_pairwise_distances_noalloc(
        dA.data_ptr(), len(A), None if dB is None else dB.data_ptr(), rows_b, A.shape[1],
        metric, p, out.data_ptr(), stream))
    torch.cuda.current_stream().synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("metric, p", [(0, 2.0), (1, 2.0), (2, 2.0), (3, 2.0), (4, 3.0),
                                      (5, 2.0)])
def test_matches_regular_entry_point_twice(metric, p):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(metric)
    # First call: larger inputs with two arrays; second: smaller, B = A, odd
    # sizes, so stale tiles of the first call sit in the scratch array.
    A1 = rng.standard_normal((1000, 37)).astype(np.float32)
    B1 = rng.standard_normal((700, 37)).astype(np.float32)
    A2 = rng.standard_normal((129, 5)).astype(np.float32)
    for A, B in ((A1, B1), (A2, None)):
        ours = no_alloc(torch, A, B, metric, p)
        np.testing.assert_allclose(ours, regular(A, B, metric, p), rtol=0, atol=0)


def test_rejects_inputs_beyond_the_scratch():
    torch = pytest.importorskip("torch")
    A = torch.zeros((70000, 128), device="cuda")
    out = torch.zeros((1, 1), device="cuda")
    status = _lib.lib.cuhc_pairwise_distances_noalloc(A.data_ptr(), 70000, None, 70000, 128, 0,
                                                      2.0, out.data_ptr(), None)
    assert status == -8
    assert "limit" in _lib.lib.cuhc_error_string(status).decode()
