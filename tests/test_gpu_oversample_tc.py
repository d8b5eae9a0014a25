"""Oversampling of several complex densities on the tensor cores
(oversample_fun_guru, surf_routs.f90:511-591, nd at once; 3xTF32 products,
FP32 accumulator) against the oracle's FP64 oversampling and the CUDA-core
engine, and inside the FP32 matvec.  Bars (w-weighted relative L2 per
density): CUDA cores 1e-7 (FP64 sums rounded to FP32 outputs; measured
2.6e-8); tensor cores 5e-7 (measured 4.2e-7: the hi/lo TF32 parts carry
about 22 significant bits and the tensor core sums the products in FP32,
against FP64 sums on the CUDA cores), which is why the CUDA-core engine is
the default."""
import ctypes as C

import numpy as np
import pytest

import oracle
from fmm3dbie_b200 import Plan
from fmm3dbie_b200 import _lib as L
from fmm3dbie_b200 import surface as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    import torch
    s = S.icosa_ellipsoid(2, 6, (1.0, 2.0, 3.0))
    zp = (5.0, -5.0j, 1.0)
    st = S.setup(s, 1, 1e-7, zp)
    P = Plan(1, zp, s, st.near, st.over)
    yield torch, s, st, P
    P.close()


def _oversample(torch, P, engine, sig):
    nd = sig.shape[1]
    x = torch.tensor(sig, device="cuda")
    out = torch.zeros((P.nptso, nd), dtype=torch.complex64, device="cuda")
    st = L.lib().bie_plan_oversample(P._h, engine, nd, C.c_void_p(x.data_ptr()),
                                     C.c_void_p(out.data_ptr()), C.c_void_p(0))
    L.check(st, "bie_plan_oversample")
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("nd", [16, 64])
def test_tensor_core_oversampling_matches_oracle(case, nd):
    torch, s, st, P = case
    rng = np.random.default_rng(nd)
    sig = rng.normal(size=(s.npts, nd)) + 1j * rng.normal(size=(s.npts, nd))
    ref = oracle.oversample_fun_surf(s, np.concatenate([sig.real, sig.imag], 1), st.over.novers,
                                     st.over.ixyzso)
    ref = ref[:, :nd] + 1j * ref[:, nd:]
    w = st.over.wover[:, None]
    for engine in (0, 1):
        got = _oversample(torch, P, engine, sig)
        err = np.sqrt(np.sum(w * np.abs(got - ref) ** 2, 0) / np.sum(w * np.abs(ref) ** 2, 0))
        print(f"\nnd {nd} engine {engine}: max per-density error {err.max():.2e}")
        assert err.max() < (1e-7 if engine == 0 else 5e-7)
    assert P.get_far(1, nd)[2] == 0, "tensor-core completion wait timed out"


def test_tensor_core_oversampling_in_matvec(case):
    torch, s, st, P = case
    rng = np.random.default_rng(7)
    nd = 32
    x = torch.tensor(rng.normal(size=(s.npts, nd)) + 1j * rng.normal(size=(s.npts, nd)),
                     device="cuda")
    assert L.lib().bie_get_oversample_engine() == 0
    y0 = P.matvec(x, 1)
    try:
        assert L.lib().bie_set_oversample_engine(1) == 0
        y1 = P.matvec(x, 1)
    finally:
        L.lib().bie_set_oversample_engine(0)
    torch.cuda.synchronize()
    d = float(torch.max(torch.abs(y1 - y0)) / torch.max(torch.abs(y0)))
    print(f"\nFP32 matvec, tensor-core vs CUDA-core oversampling: {d:.2e}")
    assert d < 1e-6
    assert P.get_far(1, nd)[2] == 0
