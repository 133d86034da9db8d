"""Parity of libturbid_gpu.so (through its C ABI) with the FP64 oracle.

Tolerances (relative L2 per field unless stated):
  * FP64 transforms / z-operators / Helmholtz solves: 1e-12
  * FP64 RK3 steps vs the oracle: 1e-10 (u, v, w, p, c) -- the reference-parity bar
  * FP32 transforms: 3e-6
  * mixed precision vs the FP64 GPU path: 1e-5 after the run
"""
import math

import numpy as np
import pytest

import turbid_b200 as tb
from oracle import turbid_oracle as O

pytestmark = pytest.mark.gpu

CASE_KEYS = ("nx", "ny", "nz", "lx", "ly", "nphase", "mapping", "mapping_coef", "slope", "slope_direction", "dt",
             "output_based_on_step", "reynolds", "froude", "averaged_concentration", "specific_gravity",
             "affected_by_scalar", "bc_u", "bc_v", "bc_w", "bc_p", "force_type", "force_direction",
             "force_amplitude", "schmidt", "settling", "erosion_rate", "critical_shear", "scalar_bc")


def gpu_case(cfg: O.CaseConfig, precision="fp64") -> tb.ChannelCase:
    """A case whose work is ordered on torch's current stream (the primitives are asynchronous)."""
    import torch
    gc = tb.ChannelCase(precision=precision, **{k: getattr(cfg, k) for k in CASE_KEYS})
    gc.set_stream(torch.cuda.current_stream().cuda_stream)
    return gc


def install_oracle_decompositions(gc, sol):
    decs = [sol.dec_u, sol.dec_v, sol.dec_w, sol.dec_p] + ([sol.dec_s] if sol.scalar else [])
    for w, d in enumerate(decs):
        gc.set_decomposition(w, d.E, d.Einv, d.lam, d.fbb, d.ftb, d.fbf, d.ftf)


def rel(a, b):
    return O.rel_l2(np.asarray(a), np.asarray(b))


def sediment_cfg(**kw):
    base = dict(nx=16, ny=12, nz=17, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                specific_gravity=2.65, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, schmidt=0.5,
                critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000)
    base.update(kw)
    return O.CaseConfig(**base)


# ----------------------------------------------------------------------------
# field-container primitives
# ----------------------------------------------------------------------------
# powers of two 8..1024 run the in-place radix-16 pass kernels, the other
# lengths the mixed-radix pass kernels (a prime factor above 13: one direct
# DFT pass, e.g. 158 = 2 x 79, 106 = 2 x 53, 34 = 2 x 17, 46 = 2 x 23)
@pytest.mark.parametrize("shape", [(24, 18, 9), (32, 32, 17), (3, 3, 5), (30, 20, 7), (8, 8, 3), (16, 64, 3),
                                   (1024, 16, 3), (8, 1024, 3), (128, 512, 3), (512, 24, 3), (256, 256, 129),
                                   (64, 64, 5), (256, 64, 3), (512, 128, 3), (64, 512, 3), (512, 256, 3),
                                   (158, 106, 5), (34, 46, 5)])
def test_dft_f64_matches_oracle(cuda, shape):
    import torch
    nx, ny, nz = shape
    cfg = O.CaseConfig(nx=nx, ny=ny, nz=nz, lx=3.0, ly=2.0)
    g = O.Grid(cfg)
    gc = gpu_case(cfg)
    rng = np.random.default_rng(7)
    x = rng.standard_normal((2, nz, ny, nx))
    ref = O.dft_forward(g, x)
    xd = torch.from_numpy(x).to(cuda)
    sd = torch.zeros((2, nz, g.M), dtype=torch.complex128, device=cuda)
    gc.dft_forward(xd.data_ptr(), sd.data_ptr(), 2)
    got = tb.from_slab(sd.cpu().numpy(), g.nxh, g.nyc)
    assert rel(got, ref) < 1e-13
    # backward of the spectral field
    xb = torch.zeros_like(xd)
    gc.dft_backward(sd.data_ptr(), xb.data_ptr(), 2)
    assert rel(xb.cpu().numpy(), O.dft_backward(g, ref)) < 1e-13
    gc.close()


@pytest.mark.parametrize("shape", [(24, 18, 9), (64, 48, 5), (256, 256, 4), (1024, 8, 3), (16, 512, 3),
                                   (32, 16, 3), (64, 128, 5), (512, 256, 3), (128, 64, 9), (512, 512, 3)])
def test_dft_f32_matches_oracle(cuda, shape):
    import torch
    nx, ny, nz = shape
    cfg = O.CaseConfig(nx=nx, ny=ny, nz=nz)
    g = O.Grid(cfg)
    gc = gpu_case(cfg, "mixed")
    x = np.random.default_rng(8).standard_normal((3, nz, ny, nx))
    ref = O.dft_forward(g, x)
    xd = torch.from_numpy(x.astype(np.float32)).to(cuda)
    sd = torch.zeros((3, nz, g.M), dtype=torch.complex128, device=cuda)
    gc.dft_forward(xd.data_ptr(), sd.data_ptr(), 3, fp32=True)
    assert rel(tb.from_slab(sd.cpu().numpy(), g.nxh, g.nyc), ref) < 3e-6
    xb = torch.zeros_like(xd)
    gc.dft_backward(sd.data_ptr(), xb.data_ptr(), 3, fp32=True)
    assert rel(xb.cpu().numpy().astype(np.float64), O.dft_backward(g, ref)) < 3e-6
    gc.close()


@pytest.mark.parametrize("nz", [9, 33, 65, 129])
def test_multiply_matches_oracle(cuda, nz):
    import torch
    cfg = O.CaseConfig(nx=12, ny=9, nz=nz)
    g = O.Grid(cfg)
    gc = gpu_case(cfg)
    rng = np.random.default_rng(9)
    A = rng.standard_normal((nz, nz))
    X = rng.standard_normal((3, g.nxh, g.nyc, nz)) + 1j * rng.standard_normal((3, g.nxh, g.nyc, nz))
    ref = O.zmul(A, X)
    xd = torch.from_numpy(tb.to_slab(X)).to(cuda)
    yd = torch.zeros_like(xd)
    gc.multiply(A, xd.data_ptr(), yd.data_ptr(), 3)
    assert rel(tb.from_slab(yd.cpu().numpy(), g.nxh, g.nyc), ref) < 1e-13
    with pytest.raises(tb.TgError):
        gc.multiply(A, xd.data_ptr(), xd.data_ptr(), 3)
    gc.close()


def test_helmholtz_matches_oracle(cuda):
    import torch
    cfg = sediment_cfg(nx=12, ny=12, nz=33)
    uvw, p, phi = O.make_initial_state(cfg, seed=1, noise=1e-2)
    sol = O.OracleSolver(cfg, uvw, p, phi)
    gc = gpu_case(cfg)
    install_oracle_decompositions(gc, sol)
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
            assert rel(got, ref) < 1e-12, (w, stage)
    gc.close()


# ----------------------------------------------------------------------------
# RK3 steps
# ----------------------------------------------------------------------------
def _compare_run(cfg, nsteps, seed, noise, tol, oracle_dec=True, check_features=True, **state_kw):
    uvw, p, phi = O.make_initial_state(cfg, seed=seed, noise=noise, **state_kw)
    sol = O.OracleSolver(cfg, uvw, p, phi if cfg.nphase > 1 else None)
    gc = gpu_case(cfg)
    if oracle_dec:
        install_oracle_decompositions(gc, sol)
    gc.upload_state(uvw, p, phi if cfg.nphase > 1 else None)
    feats = np.zeros(50)
    worst = {}
    for k in range(nsteps):
        sol.run_step()
        assert gc.run_steps(1, features=feats) == 1
        gu, gp, gphi = gc.download_state()
        pairs = {"u": (gu[0], sol.uvw[0]), "v": (gu[1], sol.uvw[1]), "w": (gu[2], sol.uvw[2]),
                 "p": (gp[0], sol.p[0])}
        if cfg.nphase > 1:
            pairs["c"] = (gphi[0], sol.phi[0])
        for name, (a, b) in pairs.items():
            e = rel(a, b)
            worst[name] = max(worst.get(name, 0.0), e)
            assert e < tol, (k, name, e)
        if check_features:
            fidx = [0, 1, 2, 3, 4, 5, 6, 7, 8, 10, 11, 12, 13, 14, 15, 19, 21, 28, 29]
            ff = np.abs(feats[fidx] - sol.fglobal[fidx])
            scale = np.maximum(np.abs(sol.fglobal[fidx]), 1e-30)
            bad = [(fidx[i], feats[fidx[i]], sol.fglobal[fidx[i]]) for i in range(len(fidx))
                   if ff[i] > max(1e-9 * scale[i], 1e-14)]
            assert not bad, (k, bad)
    t = gc.get_time()
    assert t["step"] == sol.step and abs(t["time"] - sol.time) < 1e-12 and t["alternation"] == sol.alternation
    gc.close()
    return worst


def test_fp64_steps_carrier_open_top(cuda):
    cfg = O.CaseConfig(nx=24, ny=18, nz=17, reynolds=400.0, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0],
                       dt=2 * math.pi / 2000)
    _compare_run(cfg, 4, seed=2, noise=0.05, tol=1e-10)


def test_fp64_steps_carrier_channel(cuda):
    cfg = O.CaseConfig(nx=16, ny=16, nz=33, reynolds=180.0, dt=2 * math.pi / 2000)
    _compare_run(cfg, 4, seed=3, noise=0.05, tol=1e-10)


def test_fp64_steps_with_sediment(cuda):
    _compare_run(sediment_cfg(), 4, seed=4, noise=0.05, tol=1e-10)


def test_fp64_steps_with_sediment_sloped(cuda):
    cfg = sediment_cfg(slope=0.05, slope_direction=1, nx=12, ny=12, nz=17)
    _compare_run(cfg, 11, seed=5, noise=0.05, tol=1e-10)


def test_fp64_steps_prime_factor_lengths(cuda):
    """Nx = 34 (2 x 17) and Ny = 46 (2 x 23): the direct-DFT pass of the
    mixed-radix transforms in every stage."""
    _compare_run(sediment_cfg(nx=34, ny=46, nz=17), 2, seed=14, noise=0.05, tol=1e-10)


def test_fp64_steps_radix16_transforms(cuda):
    """A 64 x 64 grid runs the in-place radix-16 transforms in every stage."""
    _compare_run(sediment_cfg(nx=64, ny=64, nz=17), 2, seed=9, noise=0.05, tol=1e-10)


def filter_active_state_kw(nz):
    """A scalar whose physical values cross zero (mean 0.05, +-0.1 noise) and
    whose mean is negative on two planes: the Bartnicki filter redistributes
    on every plane and zeroes whole planes (phase_scalar_flat.cc:419-478)."""
    mean = np.full(nz, 0.05)
    mean[4] = -0.03
    mean[11] = -0.02
    return dict(scalar_mean=mean, scalar_noise=0.1)


def test_fp64_steps_positivity_filter_active(cuda):
    cfg = sediment_cfg(nx=16, ny=12, nz=17)
    _compare_run(cfg, 3, seed=13, noise=0.05, tol=1e-10, **filter_active_state_kw(cfg.nz))


@pytest.mark.parametrize("nx,ny", [(32, 32), (30, 27)])
def test_mixed_positivity_filter_active_close_to_fp64(cuda, nx, ny):
    """The FP32 filter of the mixed mode on the same zero-crossing scalar;
    30 x 27 = 810 points per plane is no whole number of four-value vectors,
    so the filter and the feature reduction take their one-value path."""
    cfg = sediment_cfg(nx=nx, ny=ny, nz=17)
    uvw, p, phi = O.make_initial_state(cfg, seed=13, noise=0.05, **filter_active_state_kw(cfg.nz))
    f64 = gpu_case(cfg, "fp64")
    mx = gpu_case(cfg, "mixed")
    for c in (f64, mx):
        c.upload_state(uvw, p, phi)
        c.run_steps(5)
    u1, p1, c1 = f64.download_state()
    u2, p2, c2 = mx.download_state()
    assert rel(c2, c1) < 1e-5 and rel(u2, u1) < 1e-5 and rel(p2, p1) < 1e-5
    f64.close()
    mx.close()


def test_fp64_steps_native_decompositions(cuda):
    """Operators built by the library's own eigen-solver (no oracle matrices)."""
    _compare_run(sediment_cfg(nz=33), 3, seed=6, noise=0.05, tol=1e-10, oracle_dec=False, check_features=False)


def test_plugin_methods_match_run_steps(cuda):
    cfg = sediment_cfg(nx=12, ny=12, nz=17)
    uvw, p, phi = O.make_initial_state(cfg, seed=7, noise=0.05)
    a = gpu_case(cfg)
    b = gpu_case(cfg)
    for c in (a, b):
        c.upload_state(uvw, p, phi)
    a.run_steps(2)
    # the same two steps through the per-stage plugin entry points
    step, t, alt = 0, 0.0, False
    for _ in range(2):
        step += 1
        t += cfg.dt
        b.set_time(step, t, cfg.dt, alt)
        for s in range(3):
            b.carrier_predict(s)
            b.carrier_correct(s)
            b.scalar_predict(s)
            b.scalar_correct(s)
        alt = not alt
    ua, pa, ca = a.download_state()
    ub, pb, cb = b.download_state()
    assert rel(ub, ua) < 1e-14 and rel(pb, pa) < 1e-14 and rel(cb, ca) < 1e-14
    with pytest.raises(tb.TgError):
        b.carrier_predict(3)
    a.close()
    b.close()


@pytest.mark.parametrize("n", [32, 64])
def test_mixed_precision_close_to_fp64(cuda, n):
    cfg = sediment_cfg(nx=n, ny=n, nz=33)
    uvw, p, phi = O.make_initial_state(cfg, seed=8, noise=0.05)
    f64 = gpu_case(cfg, "fp64")
    mx = gpu_case(cfg, "mixed")
    for c in (f64, mx):
        c.upload_state(uvw, p, phi)
        c.run_steps(20)
    u1, p1, c1 = f64.download_state()
    u2, p2, c2 = mx.download_state()
    for name, a, b in (("u", u2[0], u1[0]), ("v", u2[1], u1[1]), ("w", u2[2], u1[2]), ("p", p2, p1),
                       ("c", c2, c1)):
        assert rel(a, b) < 1e-5, (name, rel(a, b))
    f64.close()
    mx.close()


def test_errors_are_reported(cuda):
    cfg = O.CaseConfig(nx=8, ny=8, nz=9)
    gc = gpu_case(cfg)
    with pytest.raises(tb.TgError) as e:
        gc.download_state()
    assert e.value.code == 7
    with pytest.raises(tb.TgError):
        gc.scalar_predict(0)
    gc.close()
    with pytest.raises(tb.TgError):
        tb.ChannelCase(nx=8, ny=8, nz=9, nphase=3)


# ----------------------------------------------------------------------------
# post-processor
# ----------------------------------------------------------------------------
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_swirling_strength_matches_oracle(cuda, precision):
    """lambda_ci of the velocity-gradient tensor at every point (FP64 in both
    precision modes) against the oracle's numpy eigenvalues."""
    cfg = sediment_cfg(nx=32, ny=24, nz=33)
    uvw, p, phi = O.make_initial_state(cfg, seed=12, noise=0.3)
    gc = gpu_case(cfg, precision)
    gc.upload_state(uvw, p, phi)
    got = gc.swirling_strength()
    ref = O.swirling_strength(cfg, uvw)
    assert got.shape == ref.shape and ref.max() > 0.1
    assert rel(got, ref) < 1e-10
    assert np.abs(got - ref).max() < 1e-9 * ref.max()
    with pytest.raises(tb.TgError):
        tb.ChannelCase(nx=8, ny=8, nz=9).swirling_strength()   # no state loaded
    gc.close()
