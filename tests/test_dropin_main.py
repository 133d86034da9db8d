"""The reference's main program on the GPU build: libpseudospectral.so with
include/solver_channel_flat.h (FlatChannelSolver of the reference's solver
layer over the plugin classes).

The reference's main/channelflat.cc includes solver_channel_flat.h, builds a
yueliangyi::pseudospectral::leveltwo::FlatChannelSolver from (argc, argv),
calls Configure(), isConfigured() and Execute(), and links -lpseudospectral.
turbid_b200/build.py compiles that file unchanged into turbid_b200/channelflat
when a reference source tree is at hand (TURBID_REFERENCE).

CPU: the library exports the class; a main program making the same calls
compiles and links against it; the reference's own main does too when its
tree is named by TURBID_REFERENCE.
GPU: the reference's main (when built) and the same-calls main run a case
directory in the reference's layout; the restart files they write match the
FP64 oracle (1e-10 relative L2 per field), one log line per step after the
log head; gpu_precision = Mixed in [System] gives the mixed path (1e-5).
"""
import math
import os
import shutil
import subprocess

import pytest

from oracle import turbid_oracle as O
from turbid_b200 import build as tbuild
from test_plugin_cpp import sediment_cfg, write_ini

INCLUDE = os.path.abspath(tbuild.INCLUDE)
REFERENCE = os.environ.get("TURBID_REFERENCE", "")

# A main program of our own that makes the calls the reference's main makes.
SAME_CALLS_MAIN = r"""
#include <stdexcept>
#include "solver_channel_flat.h"

int main(int argc, char** argv) {
  try {
    yueliangyi::pseudospectral::leveltwo::FlatChannelSolver solver(argc, argv);
    solver.Configure();
    if (!solver.isConfigured()) return 2;
    solver.Execute();
  } catch (std::runtime_error& err) {
    std::cout << err.what() << std::endl;
    return 1;
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def pslib():
    tbuild.build()
    return tbuild.build_pseudospectral()


def _compile_main(src_path, out_path):
    cxx = shutil.which("g++") or "c++"
    cmd = [cxx, "-O2", "-std=c++17", "-I", INCLUDE, str(src_path), "-L", tbuild.HERE, "-lpseudospectral",
           "-Wl,-rpath," + tbuild.HERE, "-o", str(out_path)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(out_path)


@pytest.fixture(scope="module")
def same_calls_main(pslib, tmp_path_factory):
    d = tmp_path_factory.mktemp("main")
    (d / "main.cc").write_text(SAME_CALLS_MAIN)
    return _compile_main(d / "main.cc", d / "channelflat_same_calls")


def test_library_exports_the_solver_class(pslib):
    out = subprocess.run(["nm", "-DC", "--defined-only", pslib], capture_output=True, text=True, check=True).stdout
    for sym in ("yueliangyi::pseudospectral::leveltwo::FlatChannelSolver::FlatChannelSolver(int&, char**&)",
                "yueliangyi::pseudospectral::leveltwo::FlatChannelSolver::Configure()",
                "yueliangyi::pseudospectral::leveltwo::FlatChannelSolver::Execute()",
                "yueliangyi::pseudospectral::leveltwo::System::System(int&, char**&)"):
        assert sym in out, sym


def test_same_calls_main_links(same_calls_main):
    assert os.access(same_calls_main, os.X_OK)


@pytest.mark.skipif(not REFERENCE or not os.path.isfile(os.path.join(REFERENCE, "main", "channelflat.cc")),
                    reason="TURBID_REFERENCE does not name a reference source tree")
def test_reference_main_compiles_unchanged(pslib, tmp_path):
    _compile_main(os.path.join(REFERENCE, "main", "channelflat.cc"), tmp_path / "channelflat")


def _case_dir(tmp_path, cfg, nsteps, seed, extra_system=""):
    uvw, p, phi = O.make_initial_state(cfg, seed=seed, noise=0.05)
    write_ini(tmp_path / "configuration.ini", cfg, maxstep=nsteps, writeinterval=nsteps)
    if extra_system:
        text = (tmp_path / "configuration.ini").read_text().replace("[System]\n", "[System]\n" + extra_system + "\n")
        (tmp_path / "configuration.ini").write_text(text)
    O.write_phase_file(str(tmp_path / "0" / "phase_00_variable.dat"), [uvw, p])
    O.write_phase_file(str(tmp_path / "0" / "phase_01_variable.dat"), [phi])
    return uvw, p, phi


def _run_and_compare(exe, tmp_path, tol, mixed=False):
    nsteps = 3
    cfg = sediment_cfg()
    uvw, p, phi = _case_dir(tmp_path, cfg, nsteps, seed=31, extra_system="gpu_precision = Mixed" if mixed else "")
    r = subprocess.run([exe, "configuration.ini", "logcomputation"], capture_output=True, text=True,
                       cwd=str(tmp_path), timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    head = [l for l in lines if "FlatChannelSolver >" in l]
    assert head and ("Mixed" in head[0]) == mixed
    steps = [l.split() for l in lines if l.split() and l.split()[0].isdigit()]
    assert [int(l[0]) for l in steps] == list(range(1, nsteps + 1))
    assert (tmp_path / "logcomputation").exists()
    sol = O.OracleSolver(cfg, uvw, p, phi)
    for _ in range(nsteps):
        sol.run_step()
    gu, gp = O.read_phase_file(str(tmp_path / str(nsteps) / "phase_00_variable.dat"), [3, 1])
    (gc,) = O.read_phase_file(str(tmp_path / str(nsteps) / "phase_01_variable.dat"), [1])
    errs = {"uvw": O.rel_l2(gu, sol.uvw), "p": O.rel_l2(gp, sol.p), "c": O.rel_l2(gc, sol.phi)}
    assert max(errs.values()) < tol, errs
    assert float(steps[-1][1]) == pytest.approx(sol.time, rel=1e-12)


@pytest.mark.gpu
def test_reference_main_runs_case_directory(cuda, pslib, tmp_path):
    exe = tbuild.REF_MAIN
    if not os.path.exists(exe):
        pytest.skip("the reference's main program was not built (no reference tree when the library was built)")
    _run_and_compare(exe, tmp_path, 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True])
def test_same_calls_main_runs_case_directory(cuda, same_calls_main, tmp_path, mixed):
    _run_and_compare(same_calls_main, tmp_path, 1e-5 if mixed else 1e-10, mixed=mixed)


def test_bad_precision_key_is_rejected(same_calls_main, tmp_path):
    """An unknown gpu_precision value stops Configure before any GPU work."""
    cfg = sediment_cfg()
    _case_dir(tmp_path, cfg, 1, seed=1, extra_system="gpu_precision = half")
    r = subprocess.run([same_calls_main, "configuration.ini"], capture_output=True, text=True, cwd=str(tmp_path),
                       timeout=60)
    assert r.returncode == 1 and "gpu_precision must be FP64 or Mixed" in r.stdout
