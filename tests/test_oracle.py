"""CPU checks of the FP64 oracle against the reference's known answers.

The reference ships no unit tests; its validation is the laminar oscillatory
Stokes solution (tmtools/get_loflow.m:17-20) compared by the RMS error of the
plane-averaged u (examples/oscillatory_flow_re180_laminar/mcode/e_analysis.m:
54-58).  These tests pin the oracle on that solution and on the algebraic
identities the reference's operators satisfy.
"""
import math
import os

import numpy as np
import pytest

from oracle import turbid_oracle as O

# Root of a yueliangyi/TURBID source tree, when one is mounted (read only);
# the tests that read its example case files skip without it.
REF = os.environ.get("TURBID_REFERENCE", "")


@pytest.mark.parametrize("nz,opentop", [(65, False), (65, True), (33, False)])
def test_laminar_stokes_known_answer(nz, opentop):
    bcu = [1, 0, 0, 1, 0] if opentop else [1, 0, 1, 0, 0]
    cfg = O.CaseConfig(nx=4, ny=4, nz=nz, reynolds=180.0, dt=2 * math.pi / 12000, bc_u=bcu, bc_v=bcu)
    uvw, p, _ = O.make_initial_state(cfg, seed=0, noise=0.0)
    sol = O.OracleSolver(cfg, uvw, p)
    for _ in range(600):
        sol.run_step()
    # plane average of u in physical space (e_analysis.m) == real mean-mode coefficient
    uphys = O.dft_backward(sol.g, sol.uvw[:1])[0]
    mu = uphys.mean(axis=(1, 2))
    ua = O.stokes_profile(180.0, sol.g.gridz, sol.time, free_slip_top=opentop)
    err = np.sqrt(np.mean((mu - ua) ** 2))
    tol = 1e-6 if nz == 33 else 2e-8
    assert err < tol, err
    assert np.allclose(mu, sol.uvw[0, 0, 0].real, atol=1e-14)


def test_transform_roundtrip_drops_unpaired_mode():
    cfg = O.CaseConfig(nx=24, ny=18, nz=9)
    g = O.Grid(cfg)
    x = np.random.default_rng(1).standard_normal((2, g.nz, g.ny, g.nx))
    s = O.dft_forward(g, x)
    s2 = O.dft_forward(g, O.dft_backward(g, s))
    d = np.abs(s2 - s).max(axis=-1)
    bad = np.argwhere(d > 1e-12)
    # only the kx=0, ky=-Nyc/2 coefficient (no Hermitian partner kept) changes: halved
    assert {tuple(b[1:]) for b in bad} <= {(0, g.nyc // 2)}
    np.testing.assert_allclose(s2[:, 0, g.nyc // 2], 0.5 * s[:, 0, g.nyc // 2], rtol=1e-12, atol=1e-15)


def test_forward_transform_matches_direct_dft():
    cfg = O.CaseConfig(nx=6, ny=9, nz=3, lx=2.0, ly=3.0)
    g = O.Grid(cfg)
    rng = np.random.default_rng(2)
    x = rng.standard_normal((1, g.nz, g.ny, g.nx))
    s = O.dft_forward(g, x)
    X, Y = np.meshgrid(np.arange(g.nx), np.arange(g.ny), indexing="xy")
    for ix in range(g.nxh):
        for iy in range(g.nyc):
            ky = g.yidx[iy]
            w = np.exp(-2j * np.pi * (ix * X / g.nx + ky * Y / g.ny))
            ref = (x[0] * w).sum(axis=(1, 2)) / (g.nx * g.ny)
            np.testing.assert_allclose(s[0, ix, iy], ref, atol=1e-13)


def test_chebyshev_d1_d2_exact_on_polynomials():
    cfg = O.CaseConfig(nx=4, ny=4, nz=17)
    g = O.Grid(cfg)
    D1, D2 = O.chebyshev_d1_d2(g)
    z = g.gridz
    for k in range(0, 16):
        f = z ** k
        d1 = k * z ** (k - 1) if k > 0 else 0 * z
        d2 = k * (k - 1) * z ** (k - 2) if k > 1 else 0 * z
        np.testing.assert_allclose(D1 @ f, d1, atol=1e-9 * max(1, k * k))
        np.testing.assert_allclose(D2 @ f, d2, atol=1e-7 * max(1, k ** 4))
    np.testing.assert_allclose(D1.sum(axis=1), 0, atol=1e-12)


def test_helmholtz_solves_collocation_system():
    """Decomposition solve == direct solve of BC rows + interior rows (+ top quirk)."""
    cfg = O.CaseConfig(nx=6, ny=6, nz=25)
    g = O.Grid(cfg)
    D1, D2 = O.chebyshev_d1_d2(g)
    n = g.nz
    rng = np.random.default_rng(3)
    for bc, sig in (([1, 0, 0, 1, 0], -5e4), ([0, 1, 0, 1, 0], 0.0), ([3.0, 1.0, 3.0, 1.0], -2e4)):
        dec = O.Dz2Decomposition(g, D1, D2, bc, [sig])
        t = rng.standard_normal((g.M, n)) + 1j * rng.standard_normal((g.M, n))
        t0 = t.copy()
        y = dec.solve(t, 0, forward_fix=(sig != 0.0))
        for m in range(1, g.M):
            k2 = g.dx2[m] + g.dy2[m]
            Aop = D2 + (k2 + sig) * np.eye(n)
            A = Aop.copy()
            A[0] = dec.A[0]
            A[-1] = dec.A[-1]
            rhs = t0[m].copy()
            if sig == 0.0:
                rhs[0] = rhs[-1] = 0.0
            x = np.linalg.solve(A, rhs)
            # the reference computes the top value with the already replaced row 0
            xq = x.copy()
            xq[-1] = x[-1] + dec.ftb[0] * (x[0] - rhs[0])
            np.testing.assert_allclose(y[m], xq, rtol=1e-9, atol=1e-12 * np.abs(xq).max())


def test_restart_file_roundtrip(tmp_path):
    cfg = O.CaseConfig(nx=8, ny=6, nz=9)
    uvw, p, phi = O.make_initial_state(cfg, seed=4, noise=1e-2)
    f = tmp_path / "0" / "phase_00_variable.dat"
    O.write_phase_file(str(f), [uvw, p])
    u2, p2 = O.read_phase_file(str(f), [3, 1])
    assert np.array_equal(u2, uvw) and np.array_equal(p2, p)
    with open(f, "rb") as fh:
        assert fh.readline() == b"IOControlLevelOne\n"
        assert fh.readline() == b"ARMA_CUB_BIN_FC016\n"
        g = O.Grid(cfg)
        assert fh.readline() == f"{g.nz} {g.nyc} {3 * g.nxh}\n".encode()


def test_ini_expressions():
    assert O.eval_expr("2*pi/12000") == pytest.approx(2 * math.pi / 12000)
    assert O.eval_expr("0.448399297311834*0.0535237234845831*1E+6") == pytest.approx(
        0.448399297311834 * 0.0535237234845831 * 1e6)
    assert O.eval_expr("10.0/(0.0535237234845831/0.448399297311834)/12/4") == pytest.approx(
        10.0 / (0.0535237234845831 / 0.448399297311834) / 12 / 4)


@pytest.mark.skipif(not REF or not os.path.isdir(REF),
                    reason="TURBID_REFERENCE does not name a reference source tree")
def test_reference_example_case_files_parse():
    for ex in ("oscillatory_flow_re180_laminar", "oscillatory_flow_re800"):
        ini = O.IniFile.load(os.path.join(REF, "examples", ex, "result", "configuration.ini"))
        c = O.CaseConfig.from_ini(ini)
        assert c.lz == 2 and c.force_type == 2
    c = O.CaseConfig.from_ini(O.IniFile.load(os.path.join(REF, "examples", "oscillatory_flow_re180_laminar",
                                                          "result", "configuration.ini")))
    assert (c.nx, c.ny, c.nz) == (3, 3, 129) and c.reynolds == 180


def test_projection_divergence_and_scalar_bounds():
    cfg = O.CaseConfig(nx=12, ny=12, nz=17, nphase=2, reynolds=800., froude=1.0, averaged_concentration=1e-3,
                       bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, critical_shear=1e-3,
                       erosion_rate=1e-4)
    uvw, p, phi = O.make_initial_state(cfg, seed=5, noise=0.05)
    sol = O.OracleSolver(cfg, uvw, p, phi)
    for _ in range(3):
        sol.run_step()
    s = sol.uvw.reshape(3, sol.g.M, sol.g.nz)
    div = O.zmul(sol.D1, s[2]) + sol.g.dx1[:, None] * s[0] + sol.g.dy1[:, None] * s[1]
    # interior divergence is at the size of the D1*D1 vs D2 splitting error, far below |u'|
    assert np.abs(div[:, 1:-1]).max() < 1e-6
    assert np.all(sol._phi_phys >= 0)
    assert np.isfinite(sol.fglobal).all()


def test_positivity_filter_branches_fire():
    """On a scalar that crosses zero, with a negative mean on two planes, the
    oracle's Bartnicki filter (phase_scalar_flat.cc:419-478) leaves no negative
    value, zeroes whole planes (kill branch) and redistributes the negative
    mass onto the positive points of the other planes."""
    cfg = O.CaseConfig(nx=16, ny=12, nz=17, nphase=2, reynolds=800., froude=1.0, averaged_concentration=1e-3,
                       bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, critical_shear=2e-4,
                       erosion_rate=1e-4)
    mean = np.full(cfg.nz, 0.05)
    mean[4] = -0.03
    mean[11] = -0.02
    uvw, p, phi = O.make_initial_state(cfg, seed=13, noise=0.05, scalar_mean=mean, scalar_noise=0.1)
    sol = O.OracleSolver(cfg, uvw, p, phi)
    before = O.dft_backward(sol.g, phi)[0]
    assert (before < 0).mean() > 0.1
    sol.positivity_filter(phi)
    pp = sol._phi_phys
    assert pp.min() == 0.0
    killed = [z for z in range(cfg.nz) if np.all(pp[z] == 0)]
    assert 4 in killed and len(killed) < cfg.nz
    kept = [z for z in range(cfg.nz) if z not in killed]
    # redistribution: the plane sums of the kept planes are unchanged (mass conserved)
    np.testing.assert_allclose(pp[kept].sum(axis=(1, 2)), before[kept].sum(axis=(1, 2)), rtol=1e-12)
