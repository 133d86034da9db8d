"""CPU checks of the C ABI library: it loads, exports every declared entry
point, and its host-side operator construction (no GPU needed) matches the
oracle's restatement of ChebyshevSpaceStepper / CmDz2DecompositionCplx."""
import os
import re

import numpy as np
import pytest

import turbid_b200 as tb
from turbid_b200 import _lib
from oracle import turbid_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(tg_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_entry_points()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.exported_names())
    assert lib.tg_version() >= 1


# entry points that take a context and check it before any CUDA call
CTX_ENTRY_POINTS = ["tg_get_dims", "tg_set_stream", "tg_synchronize", "tg_get_operators", "tg_upload_state",
                    "tg_download_state", "tg_set_time", "tg_carrier_predict", "tg_carrier_correct",
                    "tg_swirling_strength", "tg_set_graphs", "tg_autotune", "tg_run_steps", "tg_profile_begin",
                    "tg_profile_end", "tg_profile_executed", "tg_features", "tg_dft_forward_f64",
                    "tg_dft_forward_f32", "tg_dft_backward_f64", "tg_dft_backward_f32", "tg_multiply",
                    "tg_helmholtz"]


@pytest.mark.parametrize("name", CTX_ENTRY_POINTS)
def test_null_context_is_refused(name):
    """A null context returns TG_ERR_ARG with a message, no GPU touched."""
    import ctypes
    lib = _lib.load()
    fn = getattr(lib, name)
    args = []
    for t in fn.argtypes:
        if t in (ctypes.c_int, ctypes.c_longlong):
            args.append(1)
        elif t is ctypes.c_double:
            args.append(0.0)
        else:
            args.append(None)
    assert fn(*args) == 3
    assert b"null context" in lib.tg_last_error()


@pytest.mark.parametrize("nz,mapping,coef", [(17, 0, 0.0), (65, 0, 0.0), (33, 1, 0.7), (33, 2, 0.9), (33, 3, 0.8)])
def test_host_operators_match_oracle(nz, mapping, coef):
    cfg = O.CaseConfig(nx=4, ny=4, nz=nz, mapping=mapping, mapping_coef=coef)
    D1r, D2r = O.chebyshev_d1_d2(O.Grid(cfg), mapping, coef)
    D1, D2 = tb.operators_host(nz, mapping, coef)
    np.testing.assert_allclose(D1, D1r, rtol=0, atol=1e-12 * np.abs(D1r).max())
    np.testing.assert_allclose(D2, D2r, rtol=0, atol=1e-11 * np.abs(D2r).max())


@pytest.mark.parametrize("nz", [17, 65, 129])
@pytest.mark.parametrize("bc", [[0, 1, 0, 1], [1, 0, 1, 0], [1, 0, 0, 1], [4e3, 1e7, 4e3, 1e7]])
def test_host_decomposition_matches_oracle(nz, bc):
    cfg = O.CaseConfig(nx=4, ny=4, nz=nz)
    g = O.Grid(cfg)
    D1, D2 = O.chebyshev_d1_d2(g)
    ref = O.Dz2Decomposition(g, D1, D2, bc, [-1e5])
    d = tb.decomposition_host(nz, bc)
    for k in ("fbb", "ftb", "fbf", "ftf"):
        np.testing.assert_allclose(d[k], getattr(ref, k), rtol=1e-9, atol=1e-12)
    for sig in (-1e5, 0.0):
        for k2 in (0.0, -3.0):
            if sig == 0.0 and k2 == 0.0 and bc[0] != 0 and bc[1] != 0:
                continue  # Robin with sigma = k = 0 is near-singular and never assembled
            def op(E, lam, Ei):
                R = np.ones(nz)
                R[1:-1] = 1.0 / ((k2 + lam[1:-1]) + sig)
                if sig == 0.0 and k2 == 0.0:
                    R[1:-1][np.abs(lam[1:-1]) < 1e-11] = 0.0
                return (E * R) @ Ei
            S = op(d["E"], d["lam"], d["Einv"])
            Sr = op(ref.E, ref.lam, ref.Einv)
            np.testing.assert_allclose(S, Sr, rtol=0, atol=1e-11 * np.abs(Sr).max())
    # the Neumann-Neumann null eigenvalue is resolved below the reference's 1e-11 threshold
    if bc == [0, 1, 0, 1]:
        assert np.abs(d["lam"][1:-1]).min() < 1e-11


def test_ini_parser_matches_oracle():
    text = """
[System]
total_phase_number = 2
[Domain]
grid_point_number = 24 18 17
dimensionless_length = 4*pi 2*pi 2
top_bottom_slope = 0
slope_direction = 0
[Space Stepper]
applied_stepper_type = Chebyshev
mapping_function = None   # comment
mapping_coefficient = 0
[Time Stepper]
applied_stepper_type = RungeKutta3
maximum_cfl_number = 0.5
output_based_on_step = 1
maximum_task_step = 10
result_write_interval = 5
marching_time_step = 2*pi/2000
task_start_step = 0
[Phase Carrier]
applied_force_type = Oscillatory
force_direction = 0 1
force_amplitude = 0 1
reynolds_number = 800
froude_number = 1
averaged_concentration = 1e-3
specific_gravity = 2.65
affected_by_scalar_phase = 1
vertical_type_u1 = 1.0 0.0 0.0 1.0 0.0
vertical_type_u2 = 1.0 0.0 0.0 1.0 0.0
vertical_type_u3 = 1.0 0.0 1.0 0.0 0.0
vertical_type_p = 0.0 1.0 0.0 1.0 0.0
[Phase Scalar]
schmidt_number = 0.5
settling_velocity = 5e-4
vertical_boundary_type = ErosionDeposition
erosion_rate = 1e-4
critical_shear_stress = 1e-3
"""
    p = tb.params_from_ini(tb.Ini(text))
    c = O.CaseConfig.from_ini(O.IniFile(text))
    for k in ("nx", "ny", "nz", "lx", "ly", "dt", "reynolds", "settling", "critical_shear", "nphase"):
        assert p[k] == pytest.approx(getattr(c, k)), k
    assert p["bc_u"] == c.bc_u and p["force_type"] == c.force_type
    case = tb.make_case(**p)
    assert case.nz == 17 and case.bc_u[3] == 1.0 and case.scalar_bc == 1
