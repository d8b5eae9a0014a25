"""What the trained warm start gains over GMRES from zero (GPU).

A small torus of the warm-start workload's family (16 x 8 quad patches, 6 x 6
nodes, 4,608 nodes), two wavenumbers, 128 training solves per wavenumber made
by the solver itself, the network trained by the library's kernels, then
held-out directions solved from zero and from the network's guess to the
same relative residual.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KS = (2.0, 3.5)
TOL = 1e-6


@pytest.fixture(scope="module")
def trained():
    from fmm3dbie_b200.warmstart import (PlaneWaveProblem, WarmStartMLP, collect,
                                         random_directions, torus_surface, train)
    surf = torus_surface(16, 8, 5)
    prob = PlaneWaveProblem(surf, KS, eps=1e-7)
    rng = np.random.default_rng(5)
    train_dirs = {k: random_directions(128, rng) for k in KS}
    test_dirs = {k: random_directions(8, rng) for k in KS}
    dirk, tau, _ = collect(prob, train_dirs, eps=1e-7)
    mlp = WarmStartMLP(seed=5, max_rows=16384)
    losses = train(mlp, prob.srcvals, dirk, tau, steps=6000, batch=8192, lr=2e-3)
    yield prob, mlp, test_dirs, losses
    mlp.close()
    prob.close()


def _wnorm(prob, v):
    import torch
    w = torch.as_tensor(prob.surf.qwts(), device=v.device)
    return torch.sqrt((w[:, None] * v.abs() ** 2).sum(0))


def test_training_converged(trained):
    _, _, _, losses = trained
    assert np.all(np.isfinite(losses))
    assert np.mean(losses[-50:]) < 0.1 * np.mean(losses[:50])


@pytest.mark.parametrize("k", KS)
def test_warm_start_gain_mixed(trained, k):
    from fmm3dbie_b200.warmstart import PlaneWaveProblem
    prob, mlp, test_dirs, _ = trained
    d = test_dirs[k]
    dirk = PlaneWaveProblem.dirk(k, d)
    xref, iref = prob.solve(k, d, mode=0, eps=1e-11)
    x0 = mlp.predict_density(prob.srcvals, dirk)
    pred_err = (_wnorm(prob, x0 - xref) / _wnorm(prob, xref)).cpu().numpy()
    xz, iz = prob.solve(k, d, mode=1, eps=TOL)
    xw, iw = prob.solve(k, d, mode=1, eps=TOL, x0=x0)
    ez = (_wnorm(prob, xz - xref) / _wnorm(prob, xref)).cpu().numpy()
    ew = (_wnorm(prob, xw - xref) / _wnorm(prob, xref)).cpu().numpy()
    print(f"\nk={k}: prediction error {np.median(pred_err):.3e} (median); inner iterations "
          f"zero {iz['niter'].mean():.1f} warm {iw['niter'].mean():.1f}; fp64 matvecs "
          f"{iz['fp64_matvecs']} / {iw['fp64_matvecs']}; errors {ez.max():.2e} / {ew.max():.2e}")
    # both reach the tolerance (FP64 residual) and the same solution
    assert iz["status"] == 0 and iw["status"] == 0
    assert np.all(iz["rres"] <= TOL) and np.all(iw["rres"] <= TOL)
    assert ez.max() < 1e-4 and ew.max() < 1e-4
    assert not iw["x0_dropped"].any()
    assert np.median(pred_err) < 0.3 and np.all(pred_err < 0.7)
    # the gain: fewer FP32 GMRES iterations per system (GMRES gains about one
    # decade of residual per iteration here, so a guess with error e saves
    # roughly log10(1/e) iterations)
    assert iw["niter"].mean() < iz["niter"].mean()


def test_warm_start_gain_fp64(trained):
    """The reference method (FP64 GMRES) from the same guess."""
    from fmm3dbie_b200.warmstart import PlaneWaveProblem
    prob, mlp, test_dirs, _ = trained
    k = KS[0]
    d = test_dirs[k][:4]
    x0 = mlp.predict_density(prob.srcvals, PlaneWaveProblem.dirk(k, d))
    _, iz = prob.solve(k, d, mode=0, eps=TOL)
    _, iw = prob.solve(k, d, mode=0, eps=TOL, x0=x0)
    print(f"\nfp64 gmres iterations zero {iz['niter'].tolist()} warm {iw['niter'].tolist()}")
    assert np.all(iw["rres"] <= 2 * TOL) and np.all(iz["rres"] <= 2 * TOL)
    assert iw["niter"].mean() < iz["niter"].mean()


def test_bad_guess_falls_back_to_zero(trained):
    """A guess worse than zero is replaced by zero, system by system."""
    import torch
    from fmm3dbie_b200.warmstart import PlaneWaveProblem
    prob, mlp, test_dirs, _ = trained
    k = KS[1]
    d = test_dirs[k][:2]
    x0 = mlp.predict_density(prob.srcvals, PlaneWaveProblem.dirk(k, d))
    x0[:, 1] = 50.0 * torch.exp(1j * torch.arange(prob.surf.npts, device=x0.device,
                                                  dtype=torch.float64))
    _, iw = prob.solve(k, d, mode=1, eps=TOL, x0=x0.contiguous())
    assert iw["x0_dropped"].tolist() == [False, True]
    assert iw["status"] == 0 and np.all(iw["rres"] <= TOL)
