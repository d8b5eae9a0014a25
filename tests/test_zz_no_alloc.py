"""bie_farfield_dev_noalloc against bie_farfield_dev.

The no-alloc entry point serves callers that cannot allocate device memory
when they evaluate the far field (their memory belongs to their own pool or
to a fixed budget, or a cudaMalloc/cudaFree there would stall their other
streams); it takes its scratch from a fixed array in the library instead.
This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

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
    # two calls in a row, the larger first: the second (smaller) call must not
    # pick up any strength or partial sum the first call left in the array
    for seed, (ns, nt) in ((12, (5000, 1500)), (11, (3000, 700))):
        src, nrm, ch, dp, targ = problem(seed, ns, nt)
        a = run(torch, kind, zk, src, nrm, ch, dp, targ, thresh, iprec, "bie_farfield_dev")
        b = run(torch, kind, zk, src, nrm, ch, dp, targ, thresh, iprec, "bie_farfield_dev_noalloc")
        tol = 1e-12 if iprec == 0 else 2e-5
        assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(a))


def _call(kind, ns, nt):
    from fmm3dbie_b200 import _lib as L
    z = np.zeros(2)
    return L.lib().bie_farfield_dev_noalloc(kind, L.ptr(z), ns, None, None, None, None, nt, None,
                                            0.0, 1, None, C.c_void_p(0))


def test_noalloc_size_limits(torch):
    from fmm3dbie_b200 import _lib as L
    # sources: 2^20 is accepted (nt = 0 returns before any launch), one more is not
    assert _call(1, 1 << 20, 0) == 0
    assert _call(1, (1 << 20) + 1, 10) == 1
    assert b"scratch limit" in L.lib().bie_last_error()
    # targets: one chunk of partial sums must fit in 16 MiB
    assert _call(1, 10, (1 << 20) + 1) == 1
    assert b"1048576 targets" in L.lib().bie_last_error()
    assert _call(0, 10, (1 << 21) + 1) == 1
    assert b"2097152 targets" in L.lib().bie_last_error()
