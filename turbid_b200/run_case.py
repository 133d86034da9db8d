"""Run a few RK3 steps of a synthetic case on the GPU, without a case directory.

    python -m turbid_b200.run_case --nx 256 --nz 257 --steps 3 [--precision mixed]
                                   [--nphase 2] [--zsolver islice|dmma] [--seed 1234]

The case is the benchmark's oscillatory boundary layer (Re_delta = 800,
dt = 2 pi/2000, Lx = 4 pi, Ly = 2 pi, with the fine-sediment scalar unless
--nphase 1) on an Nx x Nx x Nz grid, started from the seeded synthetic state
(Stokes profile plus a divergence-free perturbation, 10 % scalar noise).  It
prints the time state after the steps; meant for quick checks and for
profiling one kernel of a known case.
"""
from __future__ import annotations

import argparse
import math

from . import synthetic
from .solver import ChannelCase


def case_params(nx: int, nz: int, nphase: int, precision: str) -> dict:
    p = dict(nx=nx, ny=nx, nz=nz, nphase=nphase, precision=precision, lx=4 * math.pi, ly=2 * math.pi,
             dt=2 * math.pi / 2000, reynolds=800.0, froude=1.0, averaged_concentration=1e-3, specific_gravity=2.65,
             affected_by_scalar=1, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], bc_w=[1, 0, 1, 0, 0],
             bc_p=[0, 1, 0, 1, 0], force_type=2, force_direction=[0, 1], force_amplitude=[0, 1], schmidt=0.5,
             settling=5e-4, erosion_rate=1e-4, critical_shear=2e-4, scalar_bc=1)
    return p


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--nx", type=int, default=64)
    ap.add_argument("--nz", type=int, default=65)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--nphase", type=int, default=2, choices=[1, 2])
    ap.add_argument("--zsolver", default=None, choices=[None, "dmma", "islice"])
    ap.add_argument("--seed", type=int, default=1234)
    args = ap.parse_args(argv)
    import torch
    p = case_params(args.nx, args.nz, args.nphase, args.precision)
    case = ChannelCase(**p)
    stream = torch.cuda.Stream()
    case.set_stream(stream.cuda_stream)
    if args.zsolver and args.precision == "mixed":
        case.set_zsolver(args.zsolver)
    uvw, pr, phi = synthetic.initial_state(seed=args.seed, **p)
    case.upload_state(uvw, pr, phi if args.nphase > 1 else None)
    case.run_steps(args.steps)
    case.synchronize()
    print(case.get_time())
    case.close()


if __name__ == "__main__":
    main()
