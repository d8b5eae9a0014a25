"""Host side of the hierarchical far field (no GPU): the cluster trees and
the dual traversal cover every (target, source) pair exactly once, for
point sets on a surface, in a volume, with coincident points and with a
single point, and the lists cost far fewer kernel evaluations than the
direct sum once the problem is large."""
import numpy as np
import pytest

from fmm3dbie_b200 import _lib as L


def _check(t, s, theta=0.5, p=8, k=0.0, leaf_t=128, leaf_s=256):
    t = np.ascontiguousarray(t, float)
    s = np.ascontiguousarray(s, float)
    out = np.zeros(14)
    st = L.lib().bie_tree_check(len(t), L.ptr(t), len(s), L.ptr(s), theta, p, k, leaf_t, leaf_s,
                                L.ptr(out))
    assert st == 0
    return out


def _ellipsoid(rng, n):
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v * np.array([1.0, 2.0, 3.0])


@pytest.mark.parametrize("theta,p,k", [(0.5, 8, 0.0), (0.7, 4, 0.0), (0.5, 10, 5.0),
                                       (0.3, 6, 0.0), (0.5, 10, 40.0)])
def test_coverage_surface(theta, p, k):
    rng = np.random.default_rng(1)
    out = _check(_ellipsoid(rng, 6000), _ellipsoid(rng, 9000), theta, p, k)
    assert out[0] == 0 and out[13] == 0
    assert out[3:8].sum() > 0
    # k-d splits at multiples of 32 near the median: target leaves of 64..128
    assert 64 <= out[10] and out[11] <= 128


def test_coverage_volume_and_small_leaves():
    rng = np.random.default_rng(2)
    out = _check(rng.uniform(-1, 1, (4000, 3)), rng.uniform(-1, 1, (5000, 3)), 0.6, 4,
                 leaf_t=16, leaf_s=16)
    assert out[0] == 0
    # every form appears with small grids and leaves
    assert all(out[3 + q] > 0 for q in (2, 3, 4))


def test_coincident_and_single_points():
    rng = np.random.default_rng(3)
    t = np.repeat(rng.uniform(-1, 1, (40, 3)), 3, axis=0)  # triples of coincident targets
    s = np.repeat(rng.uniform(-1, 1, (60, 3)), 5, axis=0)
    assert _check(t, s, 0.5, 4, leaf_t=8, leaf_s=8)[0] == 0
    assert _check(np.zeros((1, 3)), np.ones((1, 3)))[0] == 0
    assert _check(np.zeros((1, 3)), rng.uniform(-1, 1, (700, 3)), 0.5, 4, leaf_s=16)[0] == 0


def test_lists_cheaper_than_direct():
    rng = np.random.default_rng(4)
    out = _check(_ellipsoid(rng, 150000), _ellipsoid(rng, 250000), 0.5, 8)
    assert out[0] == 0
    frac = out[8] / out[9]
    print(f"\nkernel evaluations of the lists: {frac:.3f} of the direct sum")
    assert frac < 0.3


def test_high_frequency_splits_capped_nodes():
    """At k = 40 the grids of the large nodes would exceed 16 points per side:
    those nodes get no proxies and their pairs are split until the grids fit
    (on this point set down to the leaves: the lists become the direct sum,
    exact rather than under-resolved), with coverage still exact."""
    rng = np.random.default_rng(5)
    t, s = _ellipsoid(rng, 60000), _ellipsoid(rng, 100000)
    lo = _check(t, s, 0.5, 10, 2.0)
    hi = _check(t, s, 0.5, 10, 40.0)
    assert lo[0] == 0 and hi[0] == 0
    assert hi[12] > lo[12]  # more nodes too large for an accurate grid
    print(f"\nkernel evaluations of the lists: k = 2 {lo[8] / lo[9]:.3f}, k = 40 {hi[8] / hi[9]:.3f}")
    assert lo[8] < lo[9] and hi[8] <= hi[9]
