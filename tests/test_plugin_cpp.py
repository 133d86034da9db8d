"""The C++ plugin layer (include/turbid_plugin.hpp) through its main program
turbid_b200/channelflat_gpu, the stand-in for the reference's
main/channelflat.cc.

CPU: the program builds and links against libturbid_gpu.so; its .ini parser
and expression evaluator give the same case parameters as the Python mirror.
GPU: a case directory in the reference's layout (configuration.ini and the
restart files of task_start_step) runs for a few steps; the restart files it
writes match the FP64 oracle (1e-10 relative L2 per field, the library's own
eigen-decompositions), and it writes one log line per step.
"""
import json
import math
import os
import subprocess

import numpy as np
import pytest

import turbid_b200 as tb
from turbid_b200 import build as tbuild
from turbid_b200 import config as tconfig
from oracle import turbid_oracle as O


def _fmt(v):
    return " ".join(repr(float(x)) for x in v)


def write_ini(path, cfg: O.CaseConfig, maxstep: int, writeinterval: int, startstep: int = 0,
              lx_expr: str = None, dt_expr: str = None):
    """A configuration file with the keys the flat-channel solver reads."""
    mapping = {0: "None", 1: "TwoEndTangent", 2: "TwoEndSin", 3: "OneEndTangent"}[cfg.mapping]
    force = {0: "None", 1: "Constant", 2: "Oscillatory", 3: "Pulsatile", 4: "Damping"}[cfg.force_type]
    lines = [
        "# generated case", "[System]", f"total_phase_number = {cfg.nphase}   ; carrier (+ scalar)",
        "[Domain]", "applied_domain_type = Fixed", f"grid_point_number = {cfg.nx} {cfg.ny} {cfg.nz}",
        f"dimensionless_length = {lx_expr or repr(cfg.lx)} {repr(cfg.ly)} 2",
        f"top_bottom_slope = {cfg.slope!r}", f"slope_direction = {cfg.slope_direction}",
        "[Space Stepper]", "applied_stepper_type = Chebyshev", f"mapping_function = {mapping}",
        f"mapping_coefficient = {cfg.mapping_coef!r} 0",
        "[Time Stepper]", "applied_stepper_type = RungeKutta3", f"marching_time_step = {dt_expr or repr(cfg.dt)}",
        f"output_based_on_step = {cfg.output_based_on_step}", f"maximum_cfl_number = {cfg.maxcfl!r}",
        f"maximum_task_step = {maxstep}", f"result_write_interval = {writeinterval}", f"task_start_step = {startstep}",
        f"max_marching_time = {cfg.max_marching_time!r}", f"output_interval = {cfg.output_interval!r}",
        f"initial_time_step = {cfg.initial_time_step!r}", f"task_start_time_index = {cfg.start_time_index}",
        f"cfl_adjust_scale = {_fmt(cfg.cfl_adjust_scale)}", "result_write_initial = 0",
        "[Phase Carrier]", f"applied_force_type = {force}", f"force_direction = {cfg.force_direction[0]} {cfg.force_direction[1]}",
        f"force_amplitude = {_fmt(cfg.force_amplitude)}", f"reynolds_number = {cfg.reynolds!r}",
        f"froude_number = {cfg.froude!r}", f"averaged_concentration = {cfg.averaged_concentration!r}",
        f"specific_gravity = {cfg.specific_gravity!r}", f"affected_by_scalar_phase = {cfg.affected_by_scalar}",
        f"vertical_type_u1 = {_fmt(cfg.bc_u)}", f"vertical_type_u2 = {_fmt(cfg.bc_v)}",
        f"vertical_type_u3 = {_fmt(cfg.bc_w)}", f"vertical_type_p = {_fmt(cfg.bc_p)}",
    ]
    if cfg.nphase > 1:
        lines += ["[Phase Scalar]", f"schmidt_number = {cfg.schmidt!r}", f"settling_velocity = {cfg.settling!r}",
                  f"erosion_rate = {cfg.erosion_rate!r}",
                  "vertical_boundary_type = " + ("ErosionDeposition" if cfg.scalar_bc == 1 else "ZeroFlux"),
                  f"critical_shear_stress = {cfg.critical_shear!r} 0"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def sediment_cfg(**kw):
    base = dict(nx=16, ny=12, nz=17, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                specific_gravity=2.65, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, schmidt=0.5,
                critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000, maxcfl=1.0)
    base.update(kw)
    return O.CaseConfig(**base)


@pytest.fixture(scope="module")
def driver():
    tbuild.build()
    return tbuild.build_driver()


def test_driver_parses_like_python(driver, tmp_path):
    cfg = sediment_cfg(lx=4 * math.pi, mapping=1, mapping_coef=0.8)
    ini = tmp_path / "configuration.ini"
    write_ini(ini, cfg, maxstep=7, writeinterval=7, lx_expr="4*pi", dt_expr="2*pi/2000")
    out = subprocess.run([driver, "--parse-only", str(ini)], capture_output=True, text=True, check=True).stdout
    got = json.loads(out)
    ref = tconfig.params_from_ini(tconfig.Ini.load(str(ini)))
    for k, v in ref.items():
        if k in ("maxcfl",) or k not in got:
            continue
        if isinstance(v, list):
            np.testing.assert_allclose(got[k][:len(v)], v[:len(got[k])], rtol=1e-15, atol=0, err_msg=k)
        else:
            assert got[k] == pytest.approx(v, rel=1e-15, abs=0), k
    assert got["lx"] == 4 * math.pi and got["dt"] == 2 * math.pi / 2000
    assert got["maxstep"] == 7 and got["writeinterval"] == 7 and got["startstep"] == 0


def adaptive_cfg(**kw):
    dt0 = 2 * math.pi / 2000
    base = dict(output_based_on_step=0, initial_time_step=dt0, output_interval=2.5 * dt0,
                max_marching_time=4.2 * dt0, start_time_index=0, cfl_adjust_scale=[0.95, 0.9], maxcfl=0.05)
    base.update(kw)
    return sediment_cfg(**base)


def test_driver_parses_adaptive_keys(driver, tmp_path):
    cfg = adaptive_cfg()
    ini = tmp_path / "configuration.ini"
    write_ini(ini, cfg, maxstep=7, writeinterval=7)
    got = json.loads(subprocess.run([driver, "--parse-only", str(ini)], capture_output=True, text=True,
                                    check=True).stdout)
    ref = tconfig.params_from_ini(tconfig.Ini.load(str(ini)))
    for k in ("max_marching_time", "output_interval", "initial_time_step", "start_time_index", "dt"):
        assert got[k] == ref[k], k
    assert got["cfl_adjust_scale"] == ref["cfl_adjust_scale"] and got["dt"] == cfg.initial_time_step


@pytest.mark.parametrize("adaptive", [False, True])
def test_time_stepper_matches_oracle(driver, tmp_path, adaptive):
    """TimeStepper::Update / Update2 of the C++ layer against the oracle on a
    sequence of maximum velocity/length values (no GPU)."""
    cfg = adaptive_cfg() if adaptive else sediment_cfg(maxcfl=0.2)
    cfg.maxstep, cfg.writeinterval = 9, 3
    ini = tmp_path / "configuration.ini"
    write_ini(ini, cfg, maxstep=cfg.maxstep, writeinterval=cfg.writeinterval)
    lens = [0.0, 12.0, 30.0, 31.0, 8.0, 2.0, 55.0, 70.0, 40.0, 5.0, 5.0, 5.0]
    out = subprocess.run([driver, "--time-only", str(ini)] + [repr(v) for v in lens], capture_output=True,
                         text=True, check=True).stdout
    got = [json.loads(l) for l in out.strip().splitlines()]
    uvw, p, phi = O.make_initial_state(cfg, seed=3, noise=0.01)
    sol = O.OracleSolver(cfg, uvw, p, phi)
    ref = []
    for v in lens:
        if not sol.isforward:
            break
        sol.fglobal[19] = v
        sol.time_update() if not adaptive else sol.time_update2()
        ref.append(dict(step=sol.step, time=sol.time, dt=sol.dt, cfl=sol.cfl, forward=int(sol.isforward),
                        output=int(sol.isoutput), output_index=sol.output_time_index))
    assert len(got) == len(ref) and len(ref) >= 3
    for a, b in zip(got, ref):
        for k in ("step", "forward", "output", "output_index"):
            assert a[k] == b[k], (k, a, b)
        for k in ("time", "dt", "cfl"):
            assert a[k] == pytest.approx(b[k], rel=1e-15, abs=1e-300), (k, a, b)
    if adaptive:
        assert len({round(r["dt"], 12) for r in ref}) > 2   # dt did change


def test_driver_rejects_bad_config(driver, tmp_path):
    cfg = sediment_cfg()
    ini = tmp_path / "configuration.ini"
    write_ini(ini, cfg, maxstep=1, writeinterval=1)
    text = ini.read_text().replace("dimensionless_length = ", "dimensionless_length = 1 1 3 #")
    ini.write_text(text)
    r = subprocess.run([driver, "--parse-only", str(ini)], capture_output=True, text=True)
    assert r.returncode == 1 and "Dimensionless z-length" in r.stdout
    r = subprocess.run([driver, "--parse-only", str(tmp_path / "missing.ini")], capture_output=True, text=True)
    assert r.returncode == 1 and "IniFile::Load" in r.stdout


def test_expression_evaluator_matches_python(driver, tmp_path):
    exprs = ["2*pi/12000", "10E+6", "-2^2", "2^-1", "2^3^2", "(1+2)*3-4/5", "sqrt(2)*cos(pi/3)", "7 % 3",
             "pow(2, 10)", "exp(1)-e", "1e-3", "+4*atan(1)"]
    cfg = sediment_cfg()
    ini = tmp_path / "configuration.ini"
    for ex in exprs:
        write_ini(ini, cfg, maxstep=1, writeinterval=1, dt_expr=ex)
        out = subprocess.run([driver, "--parse-only", str(ini)], capture_output=True, text=True, check=True).stdout
        assert json.loads(out)["dt"] == pytest.approx(tconfig.expression(ex), rel=1e-15, abs=1e-300), ex


@pytest.mark.gpu
def test_driver_adaptive_dt(cuda, driver, tmp_path):
    """output_based_on_step = 0: dt follows the CFL band and lands on the output
    time; the solves are re-assembled for each dt.  The restart files of output
    time index 1 match the oracle's state at its first output."""
    cfg = adaptive_cfg()
    uvw, p, phi = O.make_initial_state(cfg, seed=22, noise=0.05)
    write_ini(tmp_path / "configuration.ini", cfg, maxstep=100, writeinterval=100)
    O.write_phase_file(str(tmp_path / "0" / "phase_00_variable.dat"), [uvw, p])
    O.write_phase_file(str(tmp_path / "0" / "phase_01_variable.dat"), [phi])
    r = subprocess.run([driver, str(tmp_path / "configuration.ini")], capture_output=True, text=True,
                       cwd=str(tmp_path), timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    sol = O.OracleSolver(cfg, uvw, p, phi)
    first = None
    dts = []
    while sol.isforward:
        sol.run_step()
        dts.append(sol.dt)
        if sol.isoutput and first is None:
            first = (sol.output_time_index, sol.uvw.copy(), sol.p.copy(), sol.phi.copy())
    assert first is not None and first[0] == 1 and len(set(dts)) > 1
    nlines = len(r.stdout.strip().splitlines())
    assert nlines == len(dts)
    gu, gp = O.read_phase_file(str(tmp_path / "1" / "phase_00_variable.dat"), [3, 1])
    (gc,) = O.read_phase_file(str(tmp_path / "1" / "phase_01_variable.dat"), [1])
    assert O.rel_l2(gu, first[1]) < 1e-10 and O.rel_l2(gp, first[2]) < 1e-10 and O.rel_l2(gc, first[3]) < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("nphase", [1, 2])
def test_driver_runs_case_directory(cuda, driver, tmp_path, nphase):
    nsteps = 3
    cfg = sediment_cfg(nphase=nphase) if nphase == 2 else O.CaseConfig(
        nx=24, ny=18, nz=17, reynolds=400.0, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], dt=2 * math.pi / 2000)
    uvw, p, phi = O.make_initial_state(cfg, seed=21, noise=0.05)
    write_ini(tmp_path / "configuration.ini", cfg, maxstep=nsteps, writeinterval=nsteps)
    O.write_phase_file(str(tmp_path / "0" / "phase_00_variable.dat"), [uvw, p])
    if nphase == 2:
        O.write_phase_file(str(tmp_path / "0" / "phase_01_variable.dat"), [phi])
    r = subprocess.run([driver, str(tmp_path / "configuration.ini")], capture_output=True, text=True,
                       cwd=str(tmp_path), timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    log = [l.split() for l in r.stdout.strip().splitlines()]
    assert [int(l[0]) for l in log] == list(range(1, nsteps + 1))
    assert (tmp_path / "logcomputation").exists()
    sol = O.OracleSolver(cfg, uvw, p, phi if nphase == 2 else None)
    for _ in range(nsteps):
        sol.run_step()
    gu, gp = O.read_phase_file(str(tmp_path / str(nsteps) / "phase_00_variable.dat"), [3, 1])
    assert O.rel_l2(gu, sol.uvw) < 1e-10 and O.rel_l2(gp, sol.p) < 1e-10
    if nphase == 2:
        (gc,) = O.read_phase_file(str(tmp_path / str(nsteps) / "phase_01_variable.dat"), [1])
        assert O.rel_l2(gc, sol.phi) < 1e-10
    # the log line carries the reference's columns: step, time, CFL, features 0..8
    assert float(log[-1][1]) == pytest.approx(sol.time, rel=1e-9)
    np.testing.assert_allclose([float(v) for v in log[-1][3:12]], sol.fglobal[0:9], rtol=1e-5, atol=1e-12)


@pytest.mark.gpu
def test_driver_postprocess(cuda, driver, tmp_path):
    """--postprocess: the states of [PostProcessor] work_index_range get their
    swirling strength written as <index>/phase_00_vortex.dat."""
    cfg = sediment_cfg()
    write_ini(tmp_path / "configuration.ini", cfg, maxstep=1, writeinterval=1)
    with open(tmp_path / "configuration.ini", "a") as f:
        f.write("[PostProcessor]\nwork_index_range = 3 4\n")
    refs = {}
    for idx in (3, 4):
        uvw, p, phi = O.make_initial_state(cfg, seed=50 + idx, noise=0.3)
        O.write_phase_file(str(tmp_path / str(idx) / "phase_00_variable.dat"), [uvw, p])
        O.write_phase_file(str(tmp_path / str(idx) / "phase_01_variable.dat"), [phi])
        refs[idx] = O.swirling_strength(cfg, uvw)
    r = subprocess.run([driver, "--postprocess", str(tmp_path / "configuration.ini")], capture_output=True,
                       text=True, cwd=str(tmp_path), timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    for idx, ref in refs.items():
        with open(tmp_path / str(idx) / "phase_00_vortex.dat", "rb") as f:
            assert f.readline().strip() == b"ARMA_CUB_BIN_FN008"
            nx, ny, nz = (int(v) for v in f.readline().split())
            got = np.frombuffer(f.read(), dtype=np.float64).reshape(nz, ny, nx)
        assert (nx, ny, nz) == (cfg.nx, cfg.ny, cfg.nz)
        assert O.rel_l2(got, ref) < 1e-10
