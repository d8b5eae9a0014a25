"""Tensor-core far field of the FP32 multi-density path (GPU): the same
matvec as the CUDA-core kernels within FP32 accuracy, for several density
counts, chunkings, wavenumbers and a target count that is not a multiple of
the 64-target tile."""
import numpy as np
import pytest

from fmm3dbie_b200 import surface as S

pytestmark = pytest.mark.gpu


def _rel(a, b, w):
    num = ((w[:, None] * (a - b).abs() ** 2).sum(0)) ** 0.5
    den = ((w[:, None] * b.abs() ** 2).sum(0)) ** 0.5
    return float((num / den).max())


@pytest.fixture(scope="module", params=[(4, 1.5), (6, 3.0 + 0.5j)], ids=["order4", "order6_ck"])
def plan(request):
    import torch
    from fmm3dbie_b200 import Plan
    norder, zk = request.param
    s = S.icosa_ellipsoid(1, norder, (1.0, 2.0, 3.0))
    zp = (zk, -1j * zk, 1.0)
    st = S.setup(s, 1, 1e-7, zp)
    P = Plan(1, zp, s, st.near, st.over)
    w = torch.tensor(s.qwts(), device="cuda")
    yield P, s, w
    P.close()


@pytest.mark.parametrize("nd", [4, 16, 24, 40, 64])
def test_tc_matches_cuda_cores(plan, nd):
    import torch
    P, s, w = plan
    g = torch.Generator(device="cpu").manual_seed(nd)
    x = (torch.randn(s.npts, nd, generator=g, dtype=torch.float64)
         + 1j * torch.randn(s.npts, nd, generator=g, dtype=torch.float64)).cuda().contiguous()
    y64 = P.matvec(x, 0)
    P.set_far(1, nd, 0, 2)
    ysimt = P.matvec(x, 1)
    for variant in (3, 4):
        if variant == 4 and nd <= 32:
            continue
        for nchunks in (1, 3):
            P.set_far(1, nd, variant, nchunks)
            ytc = P.matvec(x, 1)
            torch.cuda.synchronize()
            assert P.get_far(1, nd)[2] == 0, "tensor-core completion wait timed out"
            d_simt = _rel(ytc, ysimt, w)
            d_64 = _rel(ytc, y64, w)
            e_simt = _rel(ysimt, y64, w)
            print(f"\nnd {nd} variant {variant} chunks {nchunks}: vs CUDA cores {d_simt:.2e}, "
                  f"vs FP64 {d_64:.2e} (CUDA cores vs FP64 {e_simt:.2e})")
            assert d_simt < 2e-6
            assert d_64 < max(2.0 * e_simt, 2e-6)
