"""Split Helmholtz solves of the w and pressure decompositions.

With the same condition on both walls (w: Dirichlet, p: Neumann) the
collocation operator is centro-symmetric, so the library decomposes its even
and odd folded halves separately: every eigenvector has exact parity and the
solve runs as two half-size products on the GPU.

CPU: the library's host decomposition has exactly even columns 1..h and odd
columns h+1..n-2, and its solve operator E diag(R) Einv equals the oracle's
(numpy eigenvectors of the full operator) to 1e-10.
GPU: tg_helmholtz with the library's own decompositions (the split path for
w and p, dense for u, v and the scalar) matches the oracle's solve, 1e-10.
"""
import math

import numpy as np
import pytest

import turbid_b200 as tb
from oracle import turbid_oracle as O

BCS = {"w": [1, 0, 1, 0, 0], "p": [0, 1, 0, 1, 0]}


def cfg_for(nz, **kw):
    base = dict(nx=12, ny=12, nz=nz, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                specific_gravity=2.65, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, schmidt=0.5,
                critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000)
    base.update(kw)
    return O.CaseConfig(**base)


@pytest.mark.parametrize("nz", [9, 33, 129])
@pytest.mark.parametrize("which", ["w", "p"])
def test_library_eigenvectors_have_exact_parity(nz, which):
    d = tb.decomposition_host(nz, BCS[which])
    E, h = d["E"], (nz - 1) // 2
    J = E[::-1, :]
    assert np.array_equal(J[:, 1:h + 1], E[:, 1:h + 1])          # even interior eigenvectors
    assert np.array_equal(J[:, h + 1:nz - 1], -E[:, h + 1:nz - 1])  # odd interior eigenvectors
    Ei = d["Einv"]
    assert np.array_equal(Ei[1:h + 1, ::-1], Ei[1:h + 1, :])
    assert np.array_equal(Ei[h + 1:nz - 1, ::-1], -Ei[h + 1:nz - 1, :])


@pytest.mark.parametrize("nz", [17, 65])
@pytest.mark.parametrize("which", ["w", "p"])
def test_library_split_decomposition_matches_oracle(nz, which):
    cfg = cfg_for(nz)
    sol = O.OracleSolver(cfg, *O.make_initial_state(cfg, seed=1, noise=1e-2))
    ref = sol.dec_w if which == "w" else sol.dec_p
    mine = tb.decomposition_host(nz, BCS[which])
    for k2 in (0.0, -3.0, -900.0):
        sig = 0.0 if which == "p" else -cfg.reynolds / cfg.dt / 0.125
        R = 1.0 / (k2 + ref.lam + sig + (ref.lam == 0))
        R[0] = R[-1] = 1.0
        Rm = 1.0 / (k2 + mine["lam"] + sig + (mine["lam"] == 0))
        Rm[0] = Rm[-1] = 1.0
        if which == "p" and k2 == 0.0:   # the null mode of the Neumann problem
            R[np.abs(ref.lam) < 1e-11] = 0.0
            Rm[np.abs(mine["lam"]) < 1e-11] = 0.0
            R[0] = R[-1] = Rm[0] = Rm[-1] = 1.0
        a = ref.E @ np.diag(R) @ ref.Einv
        b = mine["E"] @ np.diag(Rm) @ mine["Einv"]
        assert O.rel_l2(b, a) < 1e-10, k2


@pytest.mark.gpu
@pytest.mark.parametrize("nz", [17, 65, 129])
def test_native_split_solves_match_oracle(cuda, nz):
    import torch
    cfg = cfg_for(nz)
    uvw, p, phi = O.make_initial_state(cfg, seed=1, noise=1e-2)
    sol = O.OracleSolver(cfg, uvw, p, phi)
    gc = tb.ChannelCase(precision="fp64", **{k: getattr(cfg, k) for k in (
        "nx", "ny", "nz", "lx", "ly", "nphase", "mapping", "mapping_coef", "slope", "slope_direction", "dt",
        "output_based_on_step", "reynolds", "froude", "averaged_concentration", "specific_gravity",
        "affected_by_scalar", "bc_u", "bc_v", "bc_w", "bc_p", "force_type", "force_direction",
        "force_amplitude", "schmidt", "settling", "erosion_rate", "critical_shear", "scalar_bc")})
    gc.set_stream(torch.cuda.current_stream().cuda_stream)
    g = sol.g
    rng = np.random.default_rng(10)
    decs = [sol.dec_u, sol.dec_v, sol.dec_w, sol.dec_p, sol.dec_s]
    for w, d in enumerate(decs):
        for stage in range(3):
            t = rng.standard_normal((g.M, g.nz)) + 1j * rng.standard_normal((g.M, g.nz))
            ref = d.solve(t.copy(), stage if w != 3 else 0, forward_fix=(w != 3))
            td = torch.from_numpy(np.ascontiguousarray(t.T)).to(cuda)
            od = torch.zeros_like(td)
            gc.helmholtz(w, stage, td.data_ptr(), od.data_ptr())
            got = od.cpu().numpy().T
            assert O.rel_l2(got, ref) < 1e-10, (w, stage)
    gc.close()
