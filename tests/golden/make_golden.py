"""Writes the golden fixtures of this directory from the FP64 oracle.

    python tests/golden/make_golden.py

The reference cannot be built or run here (MPI, P3DFFT/Fortran and MKL LAPACK
are absent), so the fixtures are outputs of the oracle (oracle/turbid_oracle.py),
itself pinned on the laminar Stokes solution and on operator identities.  They
freeze the oracle's results so that a change of the oracle or of the library
shows up as a fixture mismatch, and they let the GPU tests check the library
against stored vectors.

Fixtures (numpy .npz, complex spectral fields in the reference layout
(Nxh, Nyc, Nz) per component):
  transform_24x18x9.npz     seeded physical fields and their pruned spectra
  operators_n17.npz         Chebyshev D1, D2 (no mapping) for Nz = 17
  operators_n33_map1.npz    D1, D2 with mapping 1 (coefficient 0.9) for Nz = 33
  steps_sediment_16x12x17.npz  sediment case: initial state, E/Einv/lam/fix vectors
                            of the five decompositions, state + features after
                            steps 1, 2 and 3 (both nonlinear forms)
  steps_carrier_24x18x17.npz   carrier-only open-top case, same content
"""
import dataclasses
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import turbid_oracle as O  # noqa: E402

NSTEPS = 3


def cfg_json(cfg: O.CaseConfig) -> str:
    return json.dumps(dataclasses.asdict(cfg), sort_keys=True)


def write(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path)} bytes)")


def transform_fixture():
    cfg = O.CaseConfig(nx=24, ny=18, nz=9, lx=3.0, ly=2.0)
    g = O.Grid(cfg)
    phys = np.random.default_rng(101).standard_normal((2, g.nz, g.ny, g.nx))
    write("transform_24x18x9.npz", cfg=cfg_json(cfg), phys=phys, spec=O.dft_forward(g, phys))


def operator_fixtures():
    for n, mapping, coef, name in ((17, 0, 0.0, "operators_n17.npz"), (33, 1, 0.9, "operators_n33_map1.npz")):
        cfg = O.CaseConfig(nx=8, ny=8, nz=n, mapping=mapping, mapping_coef=coef)
        g = O.Grid(cfg)
        D1, D2 = O.chebyshev_d1_d2(g, mapping, coef)
        write(name, cfg=cfg_json(cfg), D1=D1, D2=D2, gridz=g.gridz)


def steps_fixture(cfg: O.CaseConfig, seed: int, noise: float, name: str):
    uvw, p, phi = O.make_initial_state(cfg, seed=seed, noise=noise)
    scalar = cfg.nphase > 1
    sol = O.OracleSolver(cfg, uvw, p, phi if scalar else None)
    out = dict(cfg=cfg_json(cfg), seed=seed, noise=noise, uvw0=uvw, p0=p)
    if scalar:
        out["phi0"] = phi
    decs = [sol.dec_u, sol.dec_v, sol.dec_w, sol.dec_p] + ([sol.dec_s] if scalar else [])
    for w, d in enumerate(decs):
        for key in ("E", "Einv", "lam", "fbb", "ftb", "fbf", "ftf"):
            out[f"dec{w}_{key}"] = np.asarray(getattr(d, key))
    for k in range(1, NSTEPS + 1):
        sol.run_step()
        out[f"uvw{k}"] = sol.uvw.copy()
        out[f"p{k}"] = sol.p.copy()
        if scalar:
            out[f"phi{k}"] = sol.phi.copy()
        out[f"feat{k}"] = sol.fglobal.copy()
        out[f"time{k}"] = np.array([sol.step, sol.time, float(sol.alternation)])
    write(name, **out)


def sediment_cfg():
    return O.CaseConfig(nx=16, ny=12, nz=17, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                        specific_gravity=2.65, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4,
                        schmidt=0.5, critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000)


def carrier_cfg():
    return O.CaseConfig(nx=24, ny=18, nz=17, reynolds=400.0, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0],
                        dt=2 * math.pi / 2000)


if __name__ == "__main__":
    transform_fixture()
    operator_fixtures()
    steps_fixture(sediment_cfg(), seed=11, noise=0.05, name="steps_sediment_16x12x17.npz")
    steps_fixture(carrier_cfg(), seed=12, noise=0.05, name="steps_carrier_24x18x17.npz")
