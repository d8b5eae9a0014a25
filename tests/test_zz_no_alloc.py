"""bie_farfield_dev_noalloc against bie_farfield_dev.

The no-alloc entry point serves callers that cannot allocate device memory
when they evaluate the far field (their memory belongs to their own pool or
to a fixed budget, or a cudaMalloc/cudaFree there would stall their other
streams); it takes its scratch from a fixed array in the library instead.
This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

from test_gpu_farfield import problem, run  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.mark.parametrize("kind,zk", [(0, 0j), (1, 2.0 + 0j)])
@pytest.mark.parametrize("iprec", [0, 1])
def test_noalloc_matches_allocating_entry_point(torch, kind, zk, iprec):
    thresh = 1e-14
    # two calls in a row with different inputs: the second must not see the
    # first call's scratch contents
    for seed, (ns, nt) in ((11, (3000, 700)), (12, (5000, 1500))):
        src, nrm, ch, dp, targ = problem(seed, ns, nt)
        a = run(torch, kind, zk, src, nrm, ch, dp, targ, thresh, iprec, "bie_farfield_dev")
        b = run(torch, kind, zk, src, nrm, ch, dp, targ, thresh, iprec, "bie_farfield_dev_noalloc")
        tol = 1e-12 if iprec == 0 else 2e-5
        assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(a))


def test_noalloc_rejects_oversized_calls(torch):
    import ctypes as C
    from fmm3dbie_b200 import _lib as L
    z = np.zeros(2)
    st = L.lib().bie_farfield_dev_noalloc(1, L.ptr(z), (1 << 20) + 1, None, None, None, None, 10,
                                          None, 0.0, 1, None, C.c_void_p(0))
    assert st == 1
    assert b"scratch limit" in L.lib().bie_last_error()
