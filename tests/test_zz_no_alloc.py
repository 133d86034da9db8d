"""GPU check of tg_dft_forward_f64_noalloc, the allocation-free forward
transform for callers that manage all device memory themselves and must not
have the library call cudaMalloc.  Its output must agree with the
context-based tg_dft_forward_f64 (the same pruned transform, other radix
passes) to 1e-13 relative L2 on two calls in a row, the second with a
different grid, since both calls share the library's static scratch array;
the second call is also checked against the oracle's numpy transform.  Kept
in its own file so that it is collected last.
"""
import ctypes

import numpy as np
import pytest

import turbid_b200 as tb
from oracle import turbid_oracle as O
from turbid_b200 import _lib

pytestmark = pytest.mark.gpu


def _reference_forward(torch, x, nx, ny, nz, dim):
    case = tb.ChannelCase(nx=nx, ny=ny, nz=nz)
    case.set_stream(torch.cuda.current_stream().cuda_stream)
    spec = torch.zeros((dim, nz, case.M), dtype=torch.complex128, device="cuda")
    case.dft_forward(x.data_ptr(), spec.data_ptr(), dim)
    torch.cuda.synchronize()
    case.close()
    return spec


@pytest.mark.parametrize("calls", [[(64, 32, 9, 2), (256, 128, 5, 3)]])
def test_noalloc_forward_matches_context_forward(cuda, calls):
    import torch
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(21)
    for nx, ny, nz, dim in calls:   # two calls in a row share the static scratch
        x = torch.from_numpy(rng.standard_normal((dim, nz, ny, nx))).to(cuda)
        ref = _reference_forward(torch, x, nx, ny, nz, dim)
        M = ref.shape[-1]
        out = torch.full((dim, nz, M), complex(np.nan, np.nan), dtype=torch.complex128, device=cuda)
        _lib.check(lib.tg_dft_forward_f64_noalloc(nx, ny, nz, ctypes.c_void_p(x.data_ptr()),
                                                  ctypes.c_void_p(out.data_ptr()), dim, ctypes.c_void_p(stream)))
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.isfinite(a).all()
        err = np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())
        assert err < 1e-13, (nx, ny, nz, dim, err)
    # the last call against the oracle (numpy rfft/fft, pruned, scaled 1/(Nx Ny))
    g = O.Grid(O.CaseConfig(nx=nx, ny=ny, nz=nz))
    ref_np = O.dft_forward(g, x.cpu().numpy())
    assert O.rel_l2(tb.from_slab(a, g.nxh, g.nyc), ref_np) < 1e-13


def test_noalloc_forward_rejects_unsupported_sizes(cuda):
    import torch
    lib = _lib.load()
    x = torch.zeros(8, dtype=torch.float64, device=cuda)
    for nx, ny in ((2048, 64), (64, 48), (4, 64)):
        st = lib.tg_dft_forward_f64_noalloc(nx, ny, 3, ctypes.c_void_p(x.data_ptr()),
                                            ctypes.c_void_p(x.data_ptr()), 1, None)
        assert st == _lib.TG_ERR_SHAPE
        assert b"powers of two" in lib.tg_last_error()
