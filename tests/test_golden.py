"""Checks against the committed golden fixtures (tests/golden, written by
tests/golden/make_golden.py from the FP64 oracle).

CPU: the oracle and the library's host-side set-up (Chebyshev operators, own
eigen-decomposition) reproduce the fixtures.  GPU: the library's transforms and
RK3 steps, started from the stored state, reproduce the stored results.

Tolerances (relative L2 per field): oracle rerun 1e-12; host operators 1e-13;
host decomposition action 1e-10; GPU transform 1e-13; GPU RK3 steps 1e-10 with
the stored decompositions and with the library's own.
"""
import json
import math
import os

import numpy as np
import pytest

import turbid_b200 as tb
from oracle import turbid_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STEP_FIXTURES = ["steps_sediment_16x12x17.npz", "steps_carrier_24x18x17.npz"]
CASE_KEYS = ("nx", "ny", "nz", "lx", "ly", "nphase", "mapping", "mapping_coef", "slope", "slope_direction", "dt",
             "output_based_on_step", "reynolds", "froude", "averaged_concentration", "specific_gravity",
             "affected_by_scalar", "bc_u", "bc_v", "bc_w", "bc_p", "force_type", "force_direction",
             "force_amplitude", "schmidt", "settling", "erosion_rate", "critical_shear", "scalar_bc")


def load(name):
    z = np.load(os.path.join(GOLDEN, name))
    cfg = O.CaseConfig(**json.loads(str(z["cfg"])))
    return z, cfg


def rel(a, b):
    return O.rel_l2(np.asarray(a), np.asarray(b))


# ----------------------------------------------------------------------------
# CPU
# ----------------------------------------------------------------------------
def test_golden_transform_oracle():
    z, cfg = load("transform_24x18x9.npz")
    assert rel(O.dft_forward(O.Grid(cfg), z["phys"]), z["spec"]) < 1e-14


@pytest.mark.parametrize("name", ["operators_n17.npz", "operators_n33_map1.npz"])
def test_golden_operators(name):
    z, cfg = load(name)
    D1o, D2o = O.chebyshev_d1_d2(O.Grid(cfg), cfg.mapping, cfg.mapping_coef)
    assert rel(D1o, z["D1"]) < 1e-15 and rel(D2o, z["D2"]) < 1e-15
    D1, D2 = tb.operators_host(cfg.nz, cfg.mapping, cfg.mapping_coef)
    assert rel(D1, z["D1"]) < 1e-13 and rel(D2, z["D2"]) < 1e-13


@pytest.mark.parametrize("name", STEP_FIXTURES)
def test_golden_steps_oracle(name):
    z, cfg = load(name)
    scalar = cfg.nphase > 1
    sol = O.OracleSolver(cfg, z["uvw0"], z["p0"], z["phi0"] if scalar else None)
    for k in range(1, 4):
        sol.run_step()
        assert rel(sol.uvw, z[f"uvw{k}"]) < 1e-12
        assert rel(sol.p, z[f"p{k}"]) < 1e-12
        if scalar:
            assert rel(sol.phi, z[f"phi{k}"]) < 1e-12
        np.testing.assert_allclose(sol.fglobal, z[f"feat{k}"], rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize("name", STEP_FIXTURES)
def test_golden_decompositions_library_host(name):
    """The library's own eigen-solver gives the same solve operator E diag(R) Einv."""
    z, cfg = load(name)
    sol = O.OracleSolver(cfg, z["uvw0"], z["p0"], z["phi0"] if cfg.nphase > 1 else None)
    decs = [sol.dec_u, sol.dec_v, sol.dec_w, sol.dec_p] + ([sol.dec_s] if cfg.nphase > 1 else [])
    for w, d in enumerate(decs):
        mine = tb.decomposition_host(cfg.nz, d.bc, cfg.mapping, cfg.mapping_coef)
        E, Ei, lam = z[f"dec{w}_E"], z[f"dec{w}_Einv"], z[f"dec{w}_lam"]
        for k2 in (-0.5, -37.0, -1500.0):
            sig = -cfg.reynolds / cfg.dt / 0.125
            R = 1.0 / (k2 + lam + sig)
            R[0] = R[-1] = 1.0
            ref = E @ np.diag(R) @ Ei
            Rm = 1.0 / (k2 + mine["lam"] + sig)
            Rm[0] = Rm[-1] = 1.0
            got = mine["E"] @ np.diag(Rm) @ mine["Einv"]
            assert rel(got, ref) < 1e-10, (w, k2)
        for key in ("fbb", "ftb", "fbf", "ftf"):
            np.testing.assert_allclose(mine[key], z[f"dec{w}_{key}"], rtol=1e-12, atol=1e-12)


# ----------------------------------------------------------------------------
# GPU (through the C ABI)
# ----------------------------------------------------------------------------
def gpu_case(cfg, precision="fp64"):
    import torch
    gc = tb.ChannelCase(precision=precision, **{k: getattr(cfg, k) for k in CASE_KEYS})
    gc.set_stream(torch.cuda.current_stream().cuda_stream)
    return gc


@pytest.mark.gpu
def test_golden_transform_gpu(cuda):
    import torch
    z, cfg = load("transform_24x18x9.npz")
    g = O.Grid(cfg)
    gc = gpu_case(cfg)
    xd = torch.from_numpy(z["phys"]).to(cuda)
    sd = torch.zeros((2, g.nz, g.M), dtype=torch.complex128, device=cuda)
    gc.dft_forward(xd.data_ptr(), sd.data_ptr(), 2)
    assert rel(tb.from_slab(sd.cpu().numpy(), g.nxh, g.nyc), z["spec"]) < 1e-13
    gc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", STEP_FIXTURES)
@pytest.mark.parametrize("stored_dec", [True, False])
def test_golden_steps_gpu(cuda, name, stored_dec):
    z, cfg = load(name)
    scalar = cfg.nphase > 1
    gc = gpu_case(cfg)
    if stored_dec:
        for w in range(5 if scalar else 4):
            gc.set_decomposition(w, *[z[f"dec{w}_{k}"] for k in ("E", "Einv", "lam", "fbb", "ftb", "fbf", "ftf")])
    tol = 1e-10
    gc.upload_state(z["uvw0"], z["p0"], z["phi0"] if scalar else None)
    feats = np.zeros(50)
    for k in range(1, 4):
        assert gc.run_steps(1, features=feats) == 1
        u, p, c = gc.download_state()
        assert rel(u, z[f"uvw{k}"]) < tol, (k, "uvw")
        assert rel(p, z[f"p{k}"]) < tol, (k, "p")
        if scalar:
            assert rel(c, z[f"phi{k}"]) < tol, (k, "c")
        if stored_dec:
            ref = z[f"feat{k}"]
            idx = [0, 1, 2, 3, 4, 5, 6, 7, 8, 19]
            np.testing.assert_allclose(feats[idx], ref[idx], rtol=1e-9, atol=1e-14)
        t = gc.get_time()
        step, time, alt = z[f"time{k}"]
        assert t["step"] == int(step) and abs(t["time"] - time) < 1e-12 and t["alternation"] == bool(alt)
    gc.close()
