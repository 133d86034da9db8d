"""Seeded synthetic restart states, built directly in the spectral space.

The reference takes its initial condition from restart files
(<start>/phase_00_variable.dat, phase_01_variable.dat; written by the MATLAB
tools gen_init.m / w_phase_cplx.m).  This module produces such states for the
benchmark cases without any transform:

  * mean mode of u: the laminar oscillatory profile at t = 0
    (tmtools/get_loflow.m), with the free-slip-top variant
    cosh(k(z-1))/cosh(2k) when the top is free slip;
  * a divergence-free perturbation u' = curl(psi), psi = (1-z^2)^2 times
    seeded random Fourier modes |kx|,|ky| <= `modes`; its amplitude bound
    (sum of coefficient magnitudes) equals `noise`;
  * the concentration: mean mode 1 plus seeded random coefficients in every
    kept mode (Hermitian in the kx = 0 plane) of physical rms `scalar_noise`.

Arrays use the restart layout (dim, Nxh, Nyc, Nz), z fastest.
"""
from __future__ import annotations

import math

import numpy as np


def cgl(nz: int) -> np.ndarray:
    return np.cos((nz - np.arange(nz) - 1) * np.pi / (nz - 1))


def stokes_profile(re: float, z: np.ndarray, t: float, free_slip_top: bool) -> np.ndarray:
    k = (1 + 1j) / math.sqrt(2) * math.sqrt(re)
    if free_slip_top:
        prof = 1j * (np.cosh(k * (z - 1)) / np.cosh(2 * k) - 1)
    else:
        prof = 1j * (np.cosh(k * z) / np.cosh(k) - 1)
    return np.real(prof * np.exp(1j * t))


def initial_state(nx: int, ny: int, nz: int, lx: float, ly: float, reynolds: float, bc_u, seed: int = 0,
                  noise: float = 0.05, scalar_noise: float = 0.1, modes: int = 4, **_):
    nxc, nyc = nx // 3 * 2, ny // 3 * 2
    nxh = nxc // 2 + 1
    z = cgl(nz)
    rng = np.random.default_rng(seed)
    opentop = abs(bc_u[2]) <= 1e-11 and abs(bc_u[3] - 1) <= 1e-11
    uvw = np.zeros((3, nxh, nyc, nz), dtype=np.complex128)
    env = (1 - z ** 2) ** 2
    denv = -4 * z * (1 - z ** 2)
    kx1, ky1 = 2 * math.pi / lx, 2 * math.pi / ly
    mx = min(modes, nxh - 1)
    my = min(modes, nyc // 2 - 1) if nyc >= 4 else 0
    total = 0.0
    for a in range(0, mx + 1):
        for b in range(-my, my + 1):
            if a == 0 and b <= 0:
                continue   # (0,-b) is the conjugate partner of (0,b)
            psi = (rng.standard_normal(3) + 1j * rng.standard_normal(3)) / 2
            ikx, iky = 1j * a * kx1, 1j * b * ky1
            cu = iky * psi[2] * env - psi[1] * denv
            cv = psi[0] * denv - ikx * psi[2] * env
            cw = ikx * psi[1] * env - iky * psi[0] * env
            iy = b if b >= 0 else nyc + b
            for c, v in enumerate((cu, cv, cw)):
                uvw[c, a, iy] += v
                if a == 0:
                    uvw[c, 0, (nyc - b) % nyc] += np.conj(v)
            total += np.abs(np.stack([cu, cv, cw])).max() * (2 if a == 0 else 2)
    if total > 0:
        uvw *= noise / total
    prof = stokes_profile(reynolds, z, 0.0, opentop)
    prof[0] = 0.0
    if not opentop:
        prof[-1] = 0.0
    uvw[0, 0, 0, :] += prof
    p = np.zeros((1, nxh, nyc, nz), dtype=np.complex128)
    # concentration: random coefficients, Hermitian in the kx = 0 plane
    nmodes = nxh * nyc
    sig = scalar_noise / math.sqrt(2.0 * nmodes)
    phi = (rng.standard_normal((1, nxh, nyc, nz)) + 1j * rng.standard_normal((1, nxh, nyc, nz))) * sig
    for iy in range(1, nyc):
        jy = (nyc - iy) % nyc
        if iy < jy:
            phi[0, 0, jy] = np.conj(phi[0, 0, iy])
    phi[0, 0, nyc // 2] = phi[0, 0, nyc // 2].real
    phi[0, 0, 0, :] = 1.0
    return uvw, p, phi
