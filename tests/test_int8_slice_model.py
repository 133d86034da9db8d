"""CPU model of an FP64 z-operator product assembled from exact int8 slice
products (Ozaki-style splitting: Ozaki, Ogita, Oishi, Rump, "Error-free
transformations of matrix multiplication", Numer. Algorithms 2012, with integer
slices as in Ootomo, Ozaki, Yokota, "DGEMM on integer matrix multiplication
unit", 2024), on the 257-point Chebyshev operators of the 256x256x257 case.

The operator A is split by rows and the data X by columns into s slices of
signed integers of at most 64 in magnitude, each row / column scaled by a power
of two: the first slice holds 6 bits, every further one 7.  The products of
slices p and q are exact in int32 (|sum| <= 64 * 64 * 257 per pair, at most s
pairs per diagonal p + q); each diagonal is summed exactly and the diagonals
in FP64 with weight 2^-(12+7(p+q)), over p + q < s.  Here the exact integer
products are formed with FP64 matrix products (every partial sum is an integer
below 2^53) and compared with a long-double product.

The tests pin how many slices each operator of the step needs: the Helmholtz
solve chain E (R .* (E^-1 X)) (src/phase_carrier_flat.cc:861-994) reaches
FP64's own error at 8 slices and 1e-9 at 5; the second-derivative operator D2
(src/stepper_space_chebyshev.cc:101-228), whose products cancel by about four
orders of magnitude, needs 8 slices for 1e-11 (plain FP64: 7e-13).  Through
the whole RK3 step (the oracle's products replaced): the two boundary rows of
the data must be applied exactly (the scalar's Robin rows carry 1e7-scaled
values), and then 6 slices everywhere (or 5 for the solves with D1, D2 in
FP64) meet the mixed mode's budget and 8 the FP64 mode's.
"""
import math

import numpy as np
import pytest

from oracle import turbid_oracle as O

NZ = 257


def split(M, axis, s):
    """s slices and the power-of-two scales: |M / scale| <= 1 with scale the
    least power of two at or above the row / column maximum (frexp: exact, no
    floating logarithm); every step below is exact in FP64 (power-of-two
    scalings, and the difference of a value and its nearest integer)."""
    mx = np.max(np.abs(M), axis=axis, keepdims=True)
    f, e = np.frexp(np.where(mx > 0, mx, 1.0))        # mx = f 2^e, f in [0.5, 1)
    e = np.where(f == 0.5, e - 1, e).astype(np.float64)
    r = M / 2.0 ** e
    slices = []
    q = np.rint(r * 64)
    slices.append(q)
    r = r * 64 - q
    for _ in range(1, s):
        q = np.rint(r * 128)
        slices.append(q)
        r = r * 128 - q
    for q in slices:
        assert np.max(np.abs(q)) <= 64
    return slices, 2.0 ** e


def test_split_is_exact_to_its_last_slice():
    rng = np.random.default_rng(5)
    X = rng.standard_normal((NZ, 40)) * 10.0 ** rng.uniform(-8, 8, 40)
    X[:, 0] = 2.0 ** -3                                   # exact powers of two keep their exponent
    for s in (1, 3, 5, 8):
        Xs, ex = split(X, 0, s)
        back = sum(q * 2.0 ** (-(6 + 7 * p)) for p, q in enumerate(Xs)) * ex
        # half a unit of the last slice, plus the rounding of the FP64 sum above
        # (eight slices span 55 bits)
        bound = 2.0 ** (-(6 + 7 * (s - 1)) - 1) * ex + 2.0 ** -52 * np.abs(X)
        assert np.all(np.abs(back - X) <= bound)
        assert np.all(np.abs(X / ex) <= 1.0)
    assert ex[0, 0] == 2.0 ** -3


def combine(As, Xs, s):
    """Sum over the slice pairs p + q < s as the tensor-core kernel does: the
    pairs of one diagonal d = p + q summed exactly (one int32 accumulator per
    diagonal), then the diagonals in FP64 with weight 2^-(12+7d), d ascending."""
    C = np.zeros((As[0].shape[0], Xs[0].shape[1]))
    for d in range(s):
        Dd = sum(As[p] @ Xs[d - p] for p in range(d + 1))   # exact: integers below 2^53
        assert np.max(np.abs(Dd)) < 2 ** 31                  # fits the int32 accumulator
        C = Dd * 2.0 ** (-(12 + 7 * d)) + C
    return C


def sliced_product(A, X, s):
    As, ea = split(A, 1, s)
    Xs, ex = split(X, 0, s)
    return combine(As, Xs, s) * ea * ex


def exact(A, X):
    return A.astype(np.longdouble) @ X.astype(np.longdouble)


def rel(a, b):
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(np.asarray(a, dtype=np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def setup():
    cfg = O.CaseConfig(nx=24, ny=24, nz=NZ, reynolds=800.0, dt=2 * math.pi / 2000, bc_u=[1, 0, 0, 1, 0])
    g = O.Grid(cfg)
    D1, D2 = O.chebyshev_d1_d2(g)
    sc = [-cfg.reynolds / cfg.dt / O.RK3[2, s] for s in range(3)]
    dec = O.Dz2Decomposition(g, D1, D2, cfg.bc_u, sc)
    # columns: resolved Chebyshev series (coefficients decaying to 1e-13 over the
    # 257 modes, amplitudes over six decades) plus a Stokes wall layer
    rng = np.random.default_rng(11)
    z = g.gridz
    k = np.arange(NZ)
    T = np.cos(np.outer(np.arccos(np.clip(z, -1, 1)), k))
    cols = []
    delta = math.sqrt(2 / cfg.reynolds)
    for _ in range(64):
        a = rng.standard_normal(NZ) * np.exp(-k * math.log(1e13) / (NZ - 1)) * 10.0 ** rng.uniform(-6, 0)
        cols.append(T @ a + rng.uniform() * np.exp(-(z + 1) / delta) * np.cos((z + 1) / delta))
    X = np.stack(cols, axis=1)
    R = dec.R[0][: X.shape[1]].T          # (Nz, columns): reciprocal of stage 1, one column per mode
    return D1, D2, dec.E, dec.Einv, R, X


def errors(fn, ref):
    return {s: rel(fn(s), ref) for s in range(4, 9)}


def test_slices_gain_seven_bits_each(setup):
    D1, D2, E, Ei, R, X = setup
    for A in (D1, D2, E, Ei):
        err = errors(lambda s: sliced_product(A, X, s), exact(A, X))
        for s in range(4, 8):
            floor = 1e-15 if A is not D2 else 1e-13
            if err[s + 1] > floor:
                assert err[s] / err[s + 1] > 30, (s, err)


def test_solve_chain_slice_counts(setup):
    _, _, E, Ei, R, X = setup
    X = X.copy()
    X[0] = X[-1] = 0.0    # boundary rows are the fix rows' work (E, R are the identity there)
    ref = exact(E, R.astype(np.longdouble) * exact(Ei, X))   # the whole chain in long double
    fp64 = rel(E @ (R * (Ei @ X)), ref)
    err = errors(lambda s: sliced_product(E, R * sliced_product(Ei, X, s), s), ref)
    assert err[5] < 1e-8          # mixed mode budget (fields within 1e-5 after 100 steps)
    assert err[8] < 1e-14 and err[8] < 20 * fp64   # FP64 mode: at FP64's own level


def test_derivative_slice_counts(setup):
    D1, D2, _, _, _, X = setup
    e1 = errors(lambda s: sliced_product(D1, X, s), exact(D1, X))
    e2 = errors(lambda s: sliced_product(D2, X, s), exact(D2, X))
    f2 = rel(D2 @ X, exact(D2, X))
    assert e1[6] < 1e-8 and e1[8] < 1e-12
    assert e2[7] < 1e-8 and e2[8] < 1e-10
    assert f2 < e2[8]             # plain FP64 D2 stays ahead of 8 slices



def make_sliced_zmul(s, exact_rows=True, skip=()):
    """The oracle's z-operator product (zmul) through s-slice products.  With
    exact_rows the two boundary rows of the data (z = -1, 1) are applied as an
    exact FP64 rank-2 update and only the interior rows are sliced (their
    scale then ignores boundary values: the scalar's Robin rows are scaled by
    1e7, src/common.h:55).  Operators in `skip` stay plain FP64."""
    cache = {}

    def zmul(A, X):
        if any(A is k for k in skip):
            return ORIG_ZMUL(A, X)
        hit = cache.get(id(A))
        if hit is None or hit[0] is not A:
            Ai = A.copy()
            if exact_rows:
                Ai[:, 0] = Ai[:, -1] = 0.0
            hit = cache[id(A)] = (A, split(Ai, 1, s))
        As, ea = hit[1]
        R = np.stack([X.real, X.imag])
        cols = R.reshape(-1, R.shape[-1]).T.copy()            # (Nz, columns): one z-profile per column
        bottom, top = cols[0].copy(), cols[-1].copy()
        if exact_rows:
            cols[0] = cols[-1] = 0.0
        Xs, ex = split(cols, 0, s)
        C = combine(As, Xs, s) * ea * ex
        if exact_rows:
            C += np.outer(A[:, 0], bottom) + np.outer(A[:, -1], top)
        Y = C.T.reshape(R.shape)
        return Y[0] + 1j * Y[1]

    return zmul


ORIG_ZMUL = O.zmul


def sediment_case():
    return O.CaseConfig(nx=16, ny=16, nz=NZ, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                        specific_gravity=2.65, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4,
                        schmidt=0.5, critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000)


def field_error(sol, ref):
    return max(O.rel_l2(sol.uvw, ref.uvw), O.rel_l2(sol.p, ref.p), O.rel_l2(sol.phi, ref.phi))


def test_robin_rows_need_exact_boundary_rows(monkeypatch):
    """The scalar solve's data carry the 1e7-scaled Robin rows: scaled with
    them, the interior rows of E_s's product lose about 23 bits."""
    cfg = sediment_case()
    uvw, p, phi = O.make_initial_state(cfg, seed=3, noise=0.05)
    sol = O.OracleSolver(cfg, uvw, p, phi)
    worst = {True: 0.0, False: 0.0}
    variants = {k: make_sliced_zmul(6, exact_rows=k) for k in worst}

    def probe(A, X):
        y = ORIG_ZMUL(A, X)
        if A is sol.dec_s.E:
            for k, fn in variants.items():
                ys = fn(A, X)
                e = np.linalg.norm(ys[..., 1:-1] - y[..., 1:-1]) / np.linalg.norm(y[..., 1:-1])
                worst[k] = max(worst[k], e)
        return y

    monkeypatch.setattr(O, "zmul", probe)
    sol.run_step()
    assert worst[False] > 1e-4 and worst[True] < 1e-9, worst


def test_solver_with_sliced_products(monkeypatch):
    """20 RK3 steps of the 16x16x257 sediment case with the z-operator products
    through s slices (exact boundary rows), against the FP64 oracle: every
    product at 6 slices meets the mixed budget, at 8 the FP64 one; with D1 and
    D2 kept in FP64 the solves need only 5 slices for the mixed budget."""
    cfg = sediment_case()
    uvw, p, phi = O.make_initial_state(cfg, seed=3, noise=0.05)
    nsteps = 20
    ref = O.OracleSolver(cfg, uvw, p, phi)
    for _ in range(nsteps):
        ref.run_step()
    err = {}
    for key, s, deriv_fp64 in (("all6", 6, False), ("all8", 8, False), ("solves5", 5, True)):
        sol = O.OracleSolver(cfg, uvw, p, phi)
        with monkeypatch.context() as m:
            m.setattr(O, "zmul", make_sliced_zmul(s, skip=(sol.D1, sol.D2) if deriv_fp64 else ()))
            for _ in range(nsteps):
                sol.run_step()
        err[key] = field_error(sol, ref)
    assert err["all6"] < 1e-6, err
    assert err["all8"] < 1e-9, err
    assert err["solves5"] < 2e-6, err
