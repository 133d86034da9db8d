"""The int8-slice tensor-core z-operator product (islice.cu, tcgen05.mma
kind::i8) that the mixed precision mode uses for its dense Helmholtz solves.

CPU: a numpy model of the kernel's arithmetic (the slicing rule, the exact
integer sums per slice diagonal, the FP64 combination order, the exact FP64
boundary rows) reproduces the FP64 product to about 1e-9.
GPU: tg_multiply_islice equals that model bit for bit (interior rows of at
most 256, partial 128-column tiles, boundary rows scaled by 1e7, a zero
column); a mixed-precision run with the int8-slice solves stays within the
mixed budget (1e-5) of the FP64 path, and no bounded device wait gave up; a
product whose operator copies are withheld gives up its wait, reports
TG_ERR_TIMEOUT and leaves the context usable.
"""
import ctypes
import math

import numpy as np
import pytest

import turbid_b200 as tb
from oracle import turbid_oracle as O
from turbid_b200 import _lib

S = 5
KP = 256


def _split(M, S):
    """Slices of the rows of M (each row scaled by 2^e, |row 2^-e| <= 1): the
    row on the grid 2^-(6+7(S-1)) of its scale (one rounding, ties to even),
    then its signed base-128 digits in [-64, 63] from the last slice up, the
    rest in slice 0."""
    mx = np.max(np.abs(M), axis=1)
    f, e = np.frexp(np.where(mx > 0, mx, 1.0))
    e = np.where(mx > 0, np.where(f == 0.5, e - 1, e), 0)
    n = np.rint(np.ldexp(M, -e[:, None]) * 2.0 ** (6 + 7 * (S - 1))).astype(np.int64)
    out = [None] * S
    for p in range(S - 1, 0, -1):
        d = ((n + 64) & 127) - 64
        n = (n - d) >> 7
        out[p] = d.astype(np.float64)
    out[0] = n.astype(np.float64)
    assert all(np.abs(q).max() <= 64 for q in out)
    return out, e


def islice_model(A, X):
    """The kernel's product of the real nrow x nz operator A and the real
    nz x ncol data X: interior rows 1..nz-2 through the slices, boundary rows
    in FP64, every rounding step in the kernel's order."""
    nz = A.shape[1]
    As, ae = _split(A[:, 1:nz - 1], S)
    Xs, xe = _split(X[1:nz - 1].T, S)
    acc = np.zeros((A.shape[0], X.shape[1]))
    for d in range(S):
        Dd = sum(As[p] @ Xs[d - p].T for p in range(d + 1))   # exact: integers below 2^53
        assert np.abs(Dd).max() < 2 ** 31
        acc = Dd * np.ldexp(1.0, -(12 + 7 * d)) + acc        # exact: the sum stays below 2^53 units
    interior = acc * np.ldexp(1.0, ae)[:, None] * np.ldexp(1.0, xe)[None, :]
    return (A[:, :1] * X[:1] + interior) + A[:, nz - 1:] * X[nz - 1:]


def _data(rng, nz, ncol):
    X = rng.standard_normal((nz, ncol)) * 10.0 ** rng.uniform(-6, 3, ncol)[None, :]
    X[0] *= 1e7                      # Robin-row scale on the boundary rows
    X[-1] *= 3e6
    X[:, 5] = 0.0                    # an all-zero column
    X[1:-1, 7] = 0.0                 # a column with only boundary values
    return X


@pytest.mark.parametrize("nz", [17, 65, 257])
def test_model_is_close_to_the_fp64_product(nz):
    rng = np.random.default_rng(nz)
    d = tb.decomposition_host(nz, [1, 0, 0, 1])
    X = _data(rng, nz, 300)
    for A in (d["E"], d["Einv"]):
        ref = A @ X
        got = islice_model(A, X)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-9


def _case(nx, ny, nz, precision="mixed"):
    return tb.ChannelCase(nx=nx, ny=ny, nz=nz, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                          bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, schmidt=0.5,
                          critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000, precision=precision)


@pytest.mark.gpu
@pytest.mark.parametrize("nz", [33, 257])
def test_islice_product_matches_model_bitwise(cuda, nz):
    import torch
    gc = _case(24, 18, nz)
    gc.set_stream(torch.cuda.current_stream().cuda_stream)
    lib = _lib.load()
    M = gc.M
    rng = np.random.default_rng(40 + nz)
    d = tb.decomposition_host(nz, [1, 0, 0, 1])
    dim = 2
    X = np.stack([_data(rng, nz, 2 * M) for _ in range(dim)])            # (dim, nz, 2M) real view
    xd = torch.from_numpy(X.copy()).to(cuda)
    for A in (d["Einv"], d["E"], rng.standard_normal((nz, nz)) * 10.0 ** rng.uniform(-3, 3, nz)[:, None]):
        A = np.ascontiguousarray(A)
        yd = torch.full_like(xd, float("nan"))
        _lib.check(lib.tg_multiply_islice(gc.h, A.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr()), dim))
        got = yd.cpu().numpy()
        for b in range(dim):
            ref = islice_model(A, X[b])
            assert np.array_equal(got[b], ref), (nz, b, np.abs(got[b] - ref).max())
            fp64 = A @ X[b]
            assert np.linalg.norm(got[b] - fp64) / np.linalg.norm(fp64) < 1e-8
    flag = ctypes.c_int(-1)
    _lib.check(lib.tg_zsolver_error(gc.h, ctypes.byref(flag)))
    assert flag.value == 0
    gc.close()


@pytest.mark.gpu
def test_islice_product_propagates_nan(cuda):
    """A NaN in a column's interior makes that column's output NaN (the
    slicing would otherwise drop it)."""
    import torch
    nz = 33
    gc = _case(24, 18, nz)
    gc.set_stream(torch.cuda.current_stream().cuda_stream)
    lib = _lib.load()
    M = gc.M
    rng = np.random.default_rng(3)
    X = rng.standard_normal((1, nz, 2 * M))
    X[0, 10, 3] = np.nan
    A = np.ascontiguousarray(rng.standard_normal((nz, nz)))
    xd = torch.from_numpy(X).to(cuda)
    yd = torch.zeros_like(xd)
    _lib.check(lib.tg_multiply_islice(gc.h, A.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr()), 1))
    got = yd.cpu().numpy()[0]
    assert np.isnan(got[:, 3]).all()
    assert np.isfinite(np.delete(got, 3, axis=1)).all()
    gc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("nz", [65, 257])
def test_mixed_steps_with_islice_solves(cuda, nz):
    """20 mixed-precision steps with the int8-slice solves against the FP64
    path (the mixed mode's budget, 1e-5 per field) and against the same mixed
    run on FP64 tensor-core solves (the pressure, whose Neumann solve
    amplifies the last bits of the divergence, differs most: about 1e-6)."""
    cfg = O.CaseConfig(nx=32, ny=32, nz=nz, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                       bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, schmidt=0.5,
                       critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000)
    uvw, p, phi = O.make_initial_state(cfg, seed=8, noise=0.05)
    lib = _lib.load()
    runs = {}
    for name, prec, solver in (("fp64", "fp64", 0), ("dmma", "mixed", 0), ("islice", "mixed", 1)):
        gc = _case(32, 32, nz, precision=prec)
        _lib.check(lib.tg_set_zsolver(gc.h, solver))
        gc.upload_state(uvw, p, phi)
        gc.run_steps(20)
        u, pp, c = gc.download_state()
        runs[name] = {"u": u[0], "v": u[1], "w": u[2], "p": pp, "c": c}
        flag = ctypes.c_int(-1)
        _lib.check(lib.tg_zsolver_error(gc.h, ctypes.byref(flag)))
        assert flag.value == 0
        gc.close()
    for k in runs["fp64"]:
        e64 = O.rel_l2(runs["islice"][k], runs["fp64"][k])
        emx = O.rel_l2(runs["islice"][k], runs["dmma"][k])
        assert e64 < 1e-5 and emx < 5e-6, (k, e64, emx)


@pytest.mark.gpu
def test_islice_bounded_wait_gives_up_and_context_stays_usable(cuda):
    """The failure path of the product's bounded waits, without a GPU fault:
    tg_islice_selftest runs a product whose operator copies are never issued,
    so the wait for them gives up; the kernel drains, frees its tensor memory,
    sets the flag and returns, and the call reports TG_ERR_TIMEOUT.  The flag
    is cleared after it, and the context's steps afterwards equal, bit for bit,
    those of a context that never ran the check."""
    nz = 33
    cfg = O.CaseConfig(nx=24, ny=18, nz=nz, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                       bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, schmidt=0.5,
                       critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000)
    uvw, p, phi = O.make_initial_state(cfg, seed=5, noise=0.05)
    lib = _lib.load()
    states = []
    for selftest in (False, True):
        gc = _case(24, 18, nz)
        _lib.check(lib.tg_set_zsolver(gc.h, 1))
        gc.upload_state(uvw, p, phi)
        gc.run_steps(2)
        if selftest:
            assert lib.tg_islice_selftest(gc.h) == _lib.TG_ERR_TIMEOUT
            assert b"bounded wait" in lib.tg_last_error()
            flag = ctypes.c_int(-1)
            _lib.check(lib.tg_zsolver_error(gc.h, ctypes.byref(flag)))
            assert flag.value == 0
        gc.run_steps(3)
        states.append(gc.download_state())
        gc.close()
    for a, b in zip(states[0], states[1]):
        assert np.array_equal(a, b)
