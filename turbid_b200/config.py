"""Case parameters: the reference's .ini case files -> struct tg_case.

The .ini grammar follows IniFile::Load (reference src/file_ini.cc:43-112):
`[Section]` lines, `key = value` lines, '#' and ';' comments, exact-case
section and key names.  Doubles and double vectors are arithmetic expressions
(the reference evaluates them with exprtk, src/file_ini.cc:241-292); integers
use std::stoi semantics.  The keys read are those of src/configure.h:51-118
that the flat-bottom RK3 path consumes.
"""
from __future__ import annotations

import ast
import math
import operator
import re
from typing import Dict, List

from ._lib import TG_PREC_FP64, TG_PREC_MIXED, TgCase

_BIN = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
        ast.Pow: operator.pow, ast.Mod: operator.mod}
_FN = {"sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp, "log": math.log, "sqrt": math.sqrt,
       "abs": abs, "atan": math.atan, "asin": math.asin, "acos": math.acos, "sinh": math.sinh,
       "cosh": math.cosh, "tanh": math.tanh, "pow": math.pow}
_CONST = {"pi": math.pi, "e": math.e}


def expression(text: str) -> float:
    """Value of an arithmetic expression such as '2*pi/12000' or '1E+6'."""
    def ev(n):
        if isinstance(n, ast.Expression):
            return ev(n.body)
        if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)):
            return float(n.value)
        if isinstance(n, ast.BinOp) and type(n.op) in _BIN:
            return _BIN[type(n.op)](ev(n.left), ev(n.right))
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, (ast.USub, ast.UAdd)):
            v = ev(n.operand)
            return -v if isinstance(n.op, ast.USub) else v
        if isinstance(n, ast.Name) and n.id.lower() in _CONST:
            return _CONST[n.id.lower()]
        if isinstance(n, ast.Call) and isinstance(n.func, ast.Name) and n.func.id.lower() in _FN:
            return float(_FN[n.func.id.lower()](*[ev(a) for a in n.args]))
        raise ValueError(f"IniFile::GetValueDouble > cannot evaluate {text!r}")
    return ev(ast.parse(text.strip().replace("^", "**"), mode="eval"))


class Ini:
    def __init__(self, text: str):
        self.sec: Dict[str, Dict[str, str]] = {}
        cur = ""
        for line in text.splitlines():
            m = re.search(r"[;#\[=]", line)
            if not m:
                continue
            ch = line[m.start()]
            if ch == "[":
                r = line.rfind("]")
                if r > m.start():
                    cur = line[m.start() + 1:r].strip()
                    self.sec.setdefault(cur, {})
            elif ch == "=":
                self.sec.setdefault(cur, {})[line[:m.start()].strip()] = re.split(r"[;#]", line[m.start() + 1:])[0].strip()

    @classmethod
    def load(cls, path: str) -> "Ini":
        with open(path) as f:
            return cls(f.read())

    def s(self, sec: str, key: str) -> str:
        if sec not in self.sec:
            raise KeyError(f"IniFile::GetValueString > Can not Find Section: {sec}")
        if key not in self.sec[sec]:
            raise KeyError(f"IniFile::GetValueString > Can not Find Key: {key} in Section {sec}")
        return self.sec[sec][key]

    def i(self, sec, key) -> int:
        return int(self.s(sec, key).split()[0])

    def d(self, sec, key) -> float:
        return expression(self.s(sec, key))

    def v(self, sec, key) -> List[float]:
        return [expression(t) for t in self.s(sec, key).split()]


FORCES = {"NONE": 0, "CONSTANT": 1, "OSCILLATORY": 2, "PULSATILE": 3, "DAMPING": 4}
MAPPINGS = {"NONE": 0, "TWOENDTANGENT": 1, "TWOENDSIN": 2, "ONEENDTANGENT": 3}


def params_from_ini(ini: Ini) -> dict:
    """Plain dict of tg_case fields plus the run-control keys of [Time Stepper]."""
    p = {}
    p["nx"], p["ny"], p["nz"] = (int(t) for t in ini.s("Domain", "grid_point_number").split())
    lx, ly, lz = ini.v("Domain", "dimensionless_length")
    if abs(lz - 2) > 10e-12:
        raise ValueError("Domain::Domain > Dimensionless z-length Should be Equal to Two!")
    p["lx"], p["ly"] = lx, ly
    p["slope"] = ini.d("Domain", "top_bottom_slope")
    p["slope_direction"] = ini.i("Domain", "slope_direction")
    p["nphase"] = ini.i("System", "total_phase_number")
    st = ini.s("Space Stepper", "applied_stepper_type").upper()
    if st != "CHEBYSHEV":
        raise ValueError("FlatChannelSolver > only the Chebyshev space stepper is supported")
    mf = ini.s("Space Stepper", "mapping_function").upper()
    if mf not in MAPPINGS:
        raise ValueError("SpaceStepper::Configuration::Load(IniFile) > Unsupported Mapping Function!")
    p["mapping"] = MAPPINGS[mf]
    p["mapping_coef"] = ini.v("Space Stepper", "mapping_coefficient")[0]
    tt = ini.s("Time Stepper", "applied_stepper_type").upper()
    if tt != "RUNGEKUTTA3":
        raise ValueError("FlatChannelSolver > only the RungeKutta3 time stepper is supported")
    p["dt"] = ini.d("Time Stepper", "marching_time_step")
    p["output_based_on_step"] = ini.i("Time Stepper", "output_based_on_step")
    p["maxcfl"] = ini.d("Time Stepper", "maximum_cfl_number")
    p["maxstep"] = ini.i("Time Stepper", "maximum_task_step")
    p["writeinterval"] = ini.i("Time Stepper", "result_write_interval")
    p["startstep"] = ini.i("Time Stepper", "task_start_step")
    if p["output_based_on_step"] == 0:  # adaptive dt (TimeStepper::Update2)
        p["max_marching_time"] = ini.d("Time Stepper", "max_marching_time")
        p["output_interval"] = ini.d("Time Stepper", "output_interval")
        p["initial_time_step"] = ini.d("Time Stepper", "initial_time_step")
        p["start_time_index"] = ini.i("Time Stepper", "task_start_time_index")
        p["cfl_adjust_scale"] = ini.v("Time Stepper", "cfl_adjust_scale")
        p["dt"] = p["initial_time_step"]
    s = "Phase Carrier"
    ft = ini.s(s, "applied_force_type").upper()
    if ft not in FORCES:
        raise ValueError("FlatCarrierPhase::Configuration::Load(IniFile) > Unsupported Force Type!")
    p["force_type"] = FORCES[ft]
    p["force_direction"] = [int(v) for v in ini.v(s, "force_direction")]
    p["force_amplitude"] = ini.v(s, "force_amplitude")
    p["reynolds"] = ini.d(s, "reynolds_number")
    p["froude"] = ini.d(s, "froude_number")
    p["averaged_concentration"] = ini.d(s, "averaged_concentration")
    p["specific_gravity"] = ini.d(s, "specific_gravity")
    p["affected_by_scalar"] = ini.i(s, "affected_by_scalar_phase")
    p["bc_u"] = ini.v(s, "vertical_type_u1")
    p["bc_v"] = ini.v(s, "vertical_type_u2")
    p["bc_w"] = ini.v(s, "vertical_type_u3")
    p["bc_p"] = ini.v(s, "vertical_type_p")
    if p["nphase"] > 1:
        s = "Phase Scalar"
        p["schmidt"] = ini.d(s, "schmidt_number")
        p["settling"] = ini.d(s, "settling_velocity")
        p["erosion_rate"] = ini.d(s, "erosion_rate")
        bt = ini.s(s, "vertical_boundary_type").upper()
        if bt == "ZEROFLUX":
            p["scalar_bc"] = 0
        elif bt == "EROSIONDEPOSITION":
            p["scalar_bc"] = 1
            p["critical_shear"] = ini.v(s, "critical_shear_stress")[0]
        else:
            raise ValueError("FlatScalarPhase::Configuration::Load(IniFile) > Unsupported Boundary Type!")
    return p


_DEFAULTS = dict(nx=32, ny=32, nz=33, lx=4 * math.pi, ly=2 * math.pi, nphase=1, mapping=0, mapping_coef=0.0,
                 slope=0.0, slope_direction=0, dt=2 * math.pi / 2000, output_based_on_step=1, reynolds=180.0,
                 froude=1.0, averaged_concentration=0.0, specific_gravity=2.65, affected_by_scalar=1,
                 bc_u=[1, 0, 1, 0, 0], bc_v=[1, 0, 1, 0, 0], bc_w=[1, 0, 1, 0, 0], bc_p=[0, 1, 0, 1, 0],
                 force_type=2, force_direction=[0, 1], force_amplitude=[0, 1], schmidt=0.5, settling=0.0,
                 erosion_rate=0.0, critical_shear=0.0, scalar_bc=1, precision="fp64")


def make_case(**kw) -> TgCase:
    """struct tg_case from keyword parameters (missing ones take defaults)."""
    p = dict(_DEFAULTS)
    p.update({k: v for k, v in kw.items() if k in _DEFAULTS})
    c = TgCase()
    for k in ("nx", "ny", "nz", "nphase", "mapping", "slope_direction", "output_based_on_step",
              "affected_by_scalar", "force_type", "scalar_bc"):
        setattr(c, k, int(p[k]))
    for k in ("lx", "ly", "mapping_coef", "slope", "dt", "reynolds", "froude", "averaged_concentration",
              "specific_gravity", "schmidt", "settling", "erosion_rate", "critical_shear"):
        setattr(c, k, float(p[k]))
    for k in ("bc_u", "bc_v", "bc_w", "bc_p"):
        vals = list(p[k]) + [0.0] * (5 - len(p[k]))
        getattr(c, k)[:] = [float(v) for v in vals[:5]]
    fd = list(p["force_direction"]) + [0, 0]
    c.force_direction[:] = [int(fd[0]), int(fd[1])]
    fa = list(p["force_amplitude"]) + [0.0] * 4
    c.force_amplitude[:] = [float(v) for v in fa[:4]]
    prec = p["precision"]
    c.precision = {"fp64": TG_PREC_FP64, "mixed": TG_PREC_MIXED}[prec] if isinstance(prec, str) else int(prec)
    return c
