"""Host-side guards of the step loop, driven to fire without any device fault.

* The CFL stop of TimeStepper::Update (src/stepper_time.cc:106-109): with
  CFL = max(|u|/dx + |v|/dy + |w|/dz) * dt above maximum_cfl_number the loop
  clears isForward, the step is still taken, and the run ends.  The first
  step's CFL is 0 (the features start at zero), so a limit below the second
  step's CFL stops the run after exactly two steps, in tg_run_steps and in the
  C++ main program alike, as in the oracle.
* The non-finite guard: an explicit step far above the stability limit
  (dt = 10, the oracle turns non-finite within four steps) makes the velocity
  overflow; the feature maxima keep the NaN/inf and tg_run_steps returns
  TG_ERR_NAN instead of stepping on.  NaN and inf are ordinary values to every
  kernel here (no data value is ever used as an index or a loop bound).
"""
import math
import subprocess

import numpy as np
import pytest

import turbid_b200 as tb
from oracle import turbid_oracle as O
from test_plugin_cpp import write_ini

pytestmark = pytest.mark.gpu

KEYS = ("nx", "ny", "nz", "lx", "ly", "nphase", "mapping", "mapping_coef", "slope", "slope_direction", "dt",
        "output_based_on_step", "reynolds", "froude", "averaged_concentration", "specific_gravity",
        "affected_by_scalar", "bc_u", "bc_v", "bc_w", "bc_p", "force_type", "force_direction",
        "force_amplitude", "schmidt", "settling", "erosion_rate", "critical_shear", "scalar_bc")


def small_cfg(**kw):
    base = dict(nx=16, ny=12, nz=17, nphase=2, reynolds=800.0, froude=1.0, averaged_concentration=1e-3,
                specific_gravity=2.65, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0], settling=5e-4, schmidt=0.5,
                critical_shear=2e-4, erosion_rate=1e-4, dt=2 * math.pi / 2000)
    base.update(kw)
    return O.CaseConfig(**base)


def _limit_after_first_step(cfg, uvw, p, phi):
    """A CFL limit that the second step's CFL exceeds (the first step's is 0)."""
    sol = O.OracleSolver(cfg, uvw, p, phi)
    sol.run_step()
    cfl2 = sol.fglobal[19] * cfg.dt
    assert cfl2 > 0
    return 0.5 * cfl2


def test_cfl_guard_stops_run_steps(cuda):
    cfg = small_cfg()
    uvw, p, phi = O.make_initial_state(cfg, seed=41, noise=0.05)
    cfg.maxcfl = float(_limit_after_first_step(cfg, uvw, p, phi))
    sol = O.OracleSolver(cfg, uvw, p, phi)
    while sol.isforward:
        sol.run_step()
    assert sol.step == 2
    gc = tb.ChannelCase(precision="fp64", **{k: getattr(cfg, k) for k in KEYS})
    gc.upload_state(uvw, p, phi)
    done = gc.run_steps(50, maxcfl=cfg.maxcfl)
    t = gc.get_time()
    assert done == 2 and t["step"] == 2 and not t["isforward"]
    assert t["cfl"] == pytest.approx(sol.cfl, rel=1e-9)
    u, pp, c = gc.download_state()
    assert O.rel_l2(u, sol.uvw) < 1e-10 and O.rel_l2(pp, sol.p) < 1e-10 and O.rel_l2(c, sol.phi) < 1e-10
    gc.close()


def test_cfl_guard_stops_the_main_program(cuda, tmp_path):
    """channelflat_gpu ends after the step whose CFL is above the limit and
    writes that step's restart files (the output flag is set on the stop)."""
    from turbid_b200 import build as tbuild
    tbuild.build()
    driver = tbuild.build_driver()
    cfg = small_cfg()
    uvw, p, phi = O.make_initial_state(cfg, seed=42, noise=0.05)
    cfg.maxcfl = float(_limit_after_first_step(cfg, uvw, p, phi))
    write_ini(tmp_path / "configuration.ini", cfg, maxstep=50, writeinterval=50)
    O.write_phase_file(str(tmp_path / "0" / "phase_00_variable.dat"), [uvw, p])
    O.write_phase_file(str(tmp_path / "0" / "phase_01_variable.dat"), [phi])
    r = subprocess.run([driver, str(tmp_path / "configuration.ini")], capture_output=True, text=True,
                       cwd=str(tmp_path), timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert [int(l.split()[0]) for l in r.stdout.strip().splitlines()] == [1, 2]
    assert (tmp_path / "2" / "phase_00_variable.dat").exists()
    sol = O.OracleSolver(cfg, uvw, p, phi)
    while sol.isforward:
        sol.run_step()
    gu, gp = O.read_phase_file(str(tmp_path / "2" / "phase_00_variable.dat"), [3, 1])
    assert sol.step == 2 and O.rel_l2(gu, sol.uvw) < 1e-10 and O.rel_l2(gp, sol.p) < 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nonfinite_state_stops_with_nan_status(cuda, precision):
    cfg = small_cfg(nx=8, ny=8, dt=10.0)
    uvw, p, phi = O.make_initial_state(cfg, seed=3, noise=0.05)
    gc = tb.ChannelCase(precision=precision, **{k: getattr(cfg, k) for k in KEYS})
    gc.upload_state(uvw, p, phi)
    with pytest.raises(tb.TgError) as e:
        gc.run_steps(40)
    assert e.value.code == 4
    assert "non-finite" in str(e.value)
    steps = gc.get_time()["step"]
    assert 1 <= steps < 40
    # the context is still usable: a fresh, finite state steps normally
    cfg_ok = small_cfg(nx=8, ny=8)
    gc.close()
    gc = tb.ChannelCase(precision=precision, **{k: getattr(cfg_ok, k) for k in KEYS})
    gc.upload_state(*O.make_initial_state(cfg_ok, seed=3, noise=0.05))
    feats = np.zeros(50)
    assert gc.run_steps(2, features=feats) == 2 and np.isfinite(feats).all()
    gc.close()
