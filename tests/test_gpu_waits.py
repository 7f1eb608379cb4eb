"""GPU: every device-side wait of the library is bounded.

A wait whose arrival never comes must give up, report CUHC_ERROR_TIMEOUT
(-7) and leave the context usable; the same wait with its arrival made must
complete. The missing arrival is made on purpose without any fault: a block
of a cooperative grid that returns before the NN-chain kernel's grid barrier
(the reference's chain barrier spins without a limit, nn_chain.cuh:84-170),
or an mbarrier arrival the pass kernels expect that is never made.
"""

import time

import numpy as np
import pytest

import cuhc_b200 as C
from _data import blobs
from cuhc_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TIMEOUT = -7


@pytest.mark.parametrize("kind", [0, 1], ids=["grid_barrier", "mbarrier"])
def test_wait_runs_out_and_reports(kind):
    t0 = time.perf_counter()
    assert _lib.lib.cuhc_wait_selftest(kind, 1, 20_000) == TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    assert _lib.lib.cuhc_wait_selftest(kind, 0, 20_000) == 0
    # The context is still usable: a tree afterwards is exact.
    X = blobs(600, 4, seed=kind)
    np.testing.assert_array_equal(C.linkage(X, "single"), O.single_linkage(X))
