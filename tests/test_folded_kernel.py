"""The folded z-operator product (gemm.cu, zgemm_sym_kernel) at the Chebyshev
grids' larger sizes: RealCplxCube::Multiply with a centro-symmetric (D2), a
centro-antisymmetric (D1) and random centro-(anti)symmetric operators at
Nz = 97, 129 and 257 equals the FP64 product (1e-13) on two components whose
modes fill a partial column tile.
"""
import numpy as np
import pytest

import turbid_b200 as tb
from oracle import turbid_oracle as O


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _centro(rng, nz, sgn):
    A = rng.standard_normal((nz, nz))
    return 0.5 * (A + sgn * A[::-1, ::-1])


@pytest.mark.gpu
@pytest.mark.parametrize("nz", [97, 129, 257])
def test_multiply_with_folded_operators(cuda, nz):
    import torch
    cfg = O.CaseConfig(nx=24, ny=21, nz=nz)
    g = O.Grid(cfg)
    gc = tb.ChannelCase(nx=cfg.nx, ny=cfg.ny, nz=nz)
    gc.set_stream(torch.cuda.current_stream().cuda_stream)   # the products are asynchronous
    rng = np.random.default_rng(nz)
    D1, D2 = tb.operators_host(nz)
    X = rng.standard_normal((2, g.nxh, g.nyc, nz)) + 1j * rng.standard_normal((2, g.nxh, g.nyc, nz))
    xd = torch.from_numpy(tb.to_slab(X)).to(cuda)
    for A in (D2, D1, _centro(rng, nz, +1), _centro(rng, nz, -1)):
        yd = torch.full_like(xd, float("nan"))
        gc.multiply(A, xd.data_ptr(), yd.data_ptr(), 2)
        assert rel(tb.from_slab(yd.cpu().numpy(), g.nxh, g.nyc), O.zmul(A, X)) < 1e-13
    gc.close()
