"""CPU FP64 restatement of TURBID's flat-bottom Fourier-Chebyshev RK3 substep.

TEST INFRASTRUCTURE ONLY.  This module is the oracle: the parity tests, the
`__graft_entry__.smoke()` check and the `cpu_baseline` / reference arm of
`bench.py` may import it, as the checker or as the timed CPU port.  The
product (`turbid_b200`, `libturbid_gpu.so`) never imports, links or calls it.

It restates, function by function, the reference solver `yueliangyi/TURBID`
(paths below are relative to that project):

  * grids and CFL lengths ............... src/domain.cc:292-347
  * wavenumber tables ................... src/stepper_space.cc:171-256
  * Chebyshev D1 / D2 (+ mappings) ...... src/stepper_space_chebyshev.cc:101-228
  * pruned plane transforms ............. src/cube_real_cplx.cc:525-555 with the
    P3DFFT pruning of build/ftran.F90:122-248 and build/btran.F90:137-243
    (inside dependency/p3dfft-master-edited.zip), 2/3 cut from src/base.cc:228-237
  * dense z-operators ................... src/cube_real_cplx.cc:461-513
  * Helmholtz decomposition ............. src/cmdz2_decomposition.cc:19-297
  * carrier phase ....................... src/phase_carrier_flat.cc:178-994
  * carrier boundary .................... src/boundary_carrier_flat.cc:131-269
  * scalar phase / boundary ............. src/phase_scalar_flat.cc:176-667,
                                          src/boundary_scalar_flat.cc:144-156
  * RK3 coefficients, fixed-dt update ... src/stepper_time_rk3.cc:28-31,
                                          src/stepper_time.cc:72-113, 215-246
  * driver stage loop ................... src/solver_channel_flat.cc:148-293
  * restart files ....................... src/variable_carrier_flat.cc:143-377,
                                          tmtools/w_armadillo_cplx.m:38-40

Layouts mirror the reference's Armadillo storage:
  physical real field   (dim, Nz, Ny, Nx)   -- x fastest  (dcube(Nx,Ny,Nz*dim))
  spectral complex field (dim, Nxh, Nyc, Nz) -- z fastest  (ccube(Nz,Nyc,Nxh*dim))
A spectral component viewed as (M, Nz) with m = ix*Nyc + iy is the transposed
cmat(Nz, M) of the reference.

Parity pin: the reference has no tests or golden vectors and cannot be built
in this container (MPI, Fortran and LAPACK are absent).  This restatement is
pinned against the reference's own known-answer validation, the laminar
oscillatory Stokes solution (tmtools/get_loflow.m:17-20 with the RMS metric of
examples/oscillatory_flow_re180_laminar/mcode/e_analysis.m:54-58), and against
operator identities; bit-level parity with the reference binary is unpinned.
"""
from __future__ import annotations

import ast
import math
import operator
import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import scipy.fft as sfft

# Column j of RK3 = stage j; rows = (c1, c2, c3).  src/stepper_time_rk3.cc:28-31
RK3 = np.array([[0.0, -5.0 / 9.0, -153.0 / 128.0],
                [1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0],
                [1.0 / 6.0, 5.0 / 24.0, 1.0 / 8.0]])
BOUNDARY_COEF_SCALE = 10e6      # src/common.h:55 (10E+6 == 1e7)
COMPARE_NUMBER_SMALL = 10e-12   # src/common.h:42 (10E-12 == 1e-11)

WORKERS = int(os.environ.get("TURBID_ORACLE_THREADS", os.cpu_count() or 1))

FORCE_TYPES = {"NONE": 0, "CONSTANT": 1, "OSCILLATORY": 2, "PULSATILE": 3, "DAMPING": 4}
MAPPINGS = {"NONE": 0, "TWOENDTANGENT": 1, "TWOENDSIN": 2, "ONEENDTANGENT": 3}


# ----------------------------------------------------------------------------
# .ini files: sections / keys as in src/file_ini.cc:43-112, values that are
# doubles are arithmetic expressions (exprtk in the reference,
# src/file_ini.cc:241-292); this is a small restricted evaluator of our own.
# ----------------------------------------------------------------------------
_BINOPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul,
           ast.Div: operator.truediv, ast.Pow: operator.pow, ast.Mod: operator.mod}
_FUNCS = {"sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp,
          "log": math.log, "sqrt": math.sqrt, "abs": abs, "atan": math.atan,
          "asin": math.asin, "acos": math.acos, "sinh": math.sinh,
          "cosh": math.cosh, "tanh": math.tanh, "pow": math.pow}
_CONSTS = {"pi": math.pi, "e": math.e}


def eval_expr(text: str) -> float:
    """Evaluate an exprtk-style arithmetic expression ('2*pi/12000', '1E+6')."""
    src = text.strip().replace("^", "**")
    tree = ast.parse(src, mode="eval")

    def ev(node):
        if isinstance(node, ast.Expression):
            return ev(node.body)
        if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)):
            return float(node.value)
        if isinstance(node, ast.BinOp) and type(node.op) in _BINOPS:
            return _BINOPS[type(node.op)](ev(node.left), ev(node.right))
        if isinstance(node, ast.UnaryOp) and isinstance(node.op, (ast.USub, ast.UAdd)):
            v = ev(node.operand)
            return -v if isinstance(node.op, ast.USub) else v
        if isinstance(node, ast.Name) and node.id.lower() in _CONSTS:
            return _CONSTS[node.id.lower()]
        if (isinstance(node, ast.Call) and isinstance(node.func, ast.Name)
                and node.func.id.lower() in _FUNCS):
            return float(_FUNCS[node.func.id.lower()](*[ev(a) for a in node.args]))
        raise ValueError(f"unsupported expression: {text!r}")

    return ev(tree)


class IniFile:
    """Sections of `key = value` lines; '#' and ';' start comments."""

    def __init__(self, text: str):
        self.sections: Dict[str, Dict[str, str]] = {}
        section = ""
        for line in text.splitlines():
            m = re.search(r"[;#\[=]", line)
            if not m:
                continue
            c = line[m.start()]
            if c == "[":
                r = line.rfind("]")
                if r > m.start():
                    section = line[m.start() + 1:r].strip()
                    self.sections.setdefault(section, {})
            elif c == "=":
                key = line[:m.start()].strip()
                val = re.split(r"[;#]", line[m.start() + 1:])[0].strip()
                self.sections.setdefault(section, {})[key] = val

    @classmethod
    def load(cls, path: str) -> "IniFile":
        with open(path) as f:
            return cls(f.read())

    def string(self, sec: str, key: str) -> str:
        if sec not in self.sections:
            raise KeyError(f"IniFile::GetValueString > Can not Find Section: {sec}")
        if key not in self.sections[sec]:
            raise KeyError(f"IniFile::GetValueString > Can not Find Key: {key} in Section {sec}")
        return self.sections[sec][key]

    def int(self, sec, key) -> int:
        return int(self.string(sec, key))

    def double(self, sec, key) -> float:
        return eval_expr(self.string(sec, key))

    def vec(self, sec, key) -> List[float]:
        return [eval_expr(t) for t in self.string(sec, key).split()]


# ----------------------------------------------------------------------------
# Case description (one .ini worth of parameters on the hot path)
# ----------------------------------------------------------------------------
@dataclass
class CaseConfig:
    nx: int = 32
    ny: int = 32
    nz: int = 33
    lx: float = 4 * math.pi
    ly: float = 2 * math.pi
    lz: float = 2.0
    nphase: int = 1
    mapping: int = 0
    mapping_coef: float = 0.0
    slope: float = 0.0
    slope_direction: int = 0
    dt: float = 2 * math.pi / 2000
    maxcfl: float = 1.0
    output_based_on_step: int = 1
    maxstep: int = 100000
    writeinterval: int = 100000
    startstep: int = 0
    reynolds: float = 180.0
    froude: float = 1.0
    averaged_concentration: float = 0.0
    specific_gravity: float = 2.65
    affected_by_scalar: int = 1
    bc_u: List[float] = field(default_factory=lambda: [1.0, 0.0, 1.0, 0.0, 0.0])
    bc_v: List[float] = field(default_factory=lambda: [1.0, 0.0, 1.0, 0.0, 0.0])
    bc_w: List[float] = field(default_factory=lambda: [1.0, 0.0, 1.0, 0.0, 0.0])
    bc_p: List[float] = field(default_factory=lambda: [0.0, 1.0, 0.0, 1.0, 0.0])
    force_type: int = 2
    force_direction: List[int] = field(default_factory=lambda: [0, 1])
    force_amplitude: List[float] = field(default_factory=lambda: [0.0, 1.0])
    schmidt: float = 0.5
    settling: float = 0.0
    erosion_rate: float = 0.0
    critical_shear: float = 0.0
    scalar_bc: int = 1   # 0 ZeroFlux, 1 ErosionDeposition (src/phase_scalar_flat.h:23-26)
    # adaptive-dt branch (output_based_on_step = 0), src/stepper_time.cc:31-37
    max_marching_time: float = 1e300
    output_interval: float = 1e300
    initial_time_step: float = 0.0
    start_time_index: int = -1
    cfl_adjust_scale: List[float] = field(default_factory=lambda: [0.95, 0.9])

    @classmethod
    def from_ini(cls, ini: IniFile) -> "CaseConfig":
        """Reads the keys of src/configure.h:51-118 the reference reads."""
        c = cls()
        size = [int(v) for v in ini.string("Domain", "grid_point_number").split()]
        c.nx, c.ny, c.nz = size
        c.lx, c.ly, c.lz = ini.vec("Domain", "dimensionless_length")
        c.slope = ini.double("Domain", "top_bottom_slope")
        c.slope_direction = ini.int("Domain", "slope_direction")
        c.nphase = ini.int("System", "total_phase_number")
        c.mapping = MAPPINGS[ini.string("Space Stepper", "mapping_function").upper()]
        c.mapping_coef = ini.vec("Space Stepper", "mapping_coefficient")[0]
        c.maxcfl = ini.double("Time Stepper", "maximum_cfl_number")
        c.output_based_on_step = ini.int("Time Stepper", "output_based_on_step")
        c.maxstep = ini.int("Time Stepper", "maximum_task_step")
        c.writeinterval = ini.int("Time Stepper", "result_write_interval")
        c.dt = ini.double("Time Stepper", "marching_time_step")
        c.startstep = ini.int("Time Stepper", "task_start_step")
        if c.output_based_on_step == 0:
            c.max_marching_time = ini.double("Time Stepper", "max_marching_time")
            c.output_interval = ini.double("Time Stepper", "output_interval")
            c.initial_time_step = ini.double("Time Stepper", "initial_time_step")
            c.start_time_index = ini.int("Time Stepper", "task_start_time_index")
            c.cfl_adjust_scale = ini.vec("Time Stepper", "cfl_adjust_scale")
        s = "Phase Carrier"
        c.force_type = FORCE_TYPES[ini.string(s, "applied_force_type").upper()]
        c.force_direction = [int(v) for v in ini.vec(s, "force_direction")]
        c.force_amplitude = ini.vec(s, "force_amplitude")
        c.reynolds = ini.double(s, "reynolds_number")
        c.froude = ini.double(s, "froude_number")
        c.averaged_concentration = ini.double(s, "averaged_concentration")
        c.specific_gravity = ini.double(s, "specific_gravity")
        c.affected_by_scalar = ini.int(s, "affected_by_scalar_phase")
        c.bc_u = ini.vec(s, "vertical_type_u1")
        c.bc_v = ini.vec(s, "vertical_type_u2")
        c.bc_w = ini.vec(s, "vertical_type_u3")
        c.bc_p = ini.vec(s, "vertical_type_p")
        if c.nphase > 1:
            s = "Phase Scalar"
            c.schmidt = ini.double(s, "schmidt_number")
            c.settling = ini.double(s, "settling_velocity")
            c.erosion_rate = ini.double(s, "erosion_rate")
            bt = ini.string(s, "vertical_boundary_type").upper()
            if bt == "ZEROFLUX":
                c.scalar_bc = 0
            elif bt == "EROSIONDEPOSITION":
                c.scalar_bc = 1
                c.critical_shear = ini.vec(s, "critical_shear_stress")[0]
            else:
                raise ValueError("FlatScalarPhase::Configuration::Load(IniFile) > Unsupported Boundary Type!")
        return c


# ----------------------------------------------------------------------------
# Grid, wavenumbers, operators
# ----------------------------------------------------------------------------
class Grid:
    """Domain + pruned spectral space + wavenumber tables."""

    def __init__(self, cfg: CaseConfig):
        if abs(cfg.lz - 2) > COMPARE_NUMBER_SMALL:       # src/domain.cc:55-58
            raise ValueError("Domain > Dimensionless z-length Should be Equal to Two!")
        self.nx, self.ny, self.nz = cfg.nx, cfg.ny, cfg.nz
        # 2/3 cut with integer arithmetic: src/base.cc:233-234, 255-258
        self.nxc = cfg.nx // 3 * 2
        self.nyc = cfg.ny // 3 * 2
        self.nxh = self.nxc // 2 + 1
        self.M = self.nyc * self.nxh
        nz = self.nz
        # src/domain.cc:304-306
        self.gridx = cfg.lx / cfg.nx * np.arange(cfg.nx)
        self.gridy = cfg.ly / cfg.ny * np.arange(cfg.ny)
        self.gridz = np.cos((nz - np.arange(nz) - 1) * np.pi / (nz - 1))
        self.lengthminx = np.diff(self.gridx).min() if cfg.nx > 1 else cfg.lx
        self.lengthminy = np.diff(self.gridy).min() if cfg.ny > 1 else cfg.ly
        # CFL length in z per plane: src/domain.cc:317-332
        self.gridlenz = self._gridlenz(self.gridz)
        # y-index map of the P3DFFT pruning: build/ftran.F90:238-248
        h = self.nyc // 2
        self.yidx = np.concatenate([np.arange(h), np.arange(cfg.ny - (self.nyc - h), cfg.ny)])
        # wavenumbers per column m = ix*nyc + iy: src/stepper_space.cc:196-213
        kx1 = 2 * np.pi / cfg.lx
        ky1 = 2 * np.pi / cfg.ly
        ix = np.arange(self.nxh)
        iy = np.arange(self.nyc)
        kx = kx1 * ix
        ky = np.where(iy <= self.nyc // 2, ky1 * iy, -ky1 * (self.nyc - iy))
        KX, KY = np.meshgrid(kx, ky, indexing="ij")
        self.kx = KX.reshape(-1)
        self.ky = KY.reshape(-1)
        self.dx1 = 1j * self.kx        # cmdx1 = (0, +kx)
        self.dy1 = 1j * self.ky        # cmdy1 = (0, +ky)
        self.dx2 = -self.kx ** 2       # cmdx2 = (-kx^2, 0)
        self.dy2 = -self.ky ** 2

    def _gridlenz(self, gz):
        nz = len(gz)
        out = np.empty(nz)
        for k in range(nz):
            if k == 0:
                out[k] = (gz[1] - gz[0]) / 2
            elif k == nz - 1:
                out[k] = (gz[nz - 1] - gz[nz - 2]) / 2
            else:
                out[k] = min(gz[k + 1] - gz[k], gz[k] - gz[k - 1])
        return out


def chebyshev_d1_d2(grid: Grid, mapping: int = 0, coef: float = 0.0):
    """Collocation D1 (negative-sum diagonal) and D2 = D1*D1 (negative-sum diagonal).

    src/stepper_space_chebyshev.cc:122-228.  With a mapping, D1 is premultiplied by
    the mapping derivative and the z CFL lengths follow the clustered grid.
    """
    z = grid.gridz
    n = len(z)
    D = np.zeros((n, n))
    i, j = np.tril_indices(n, -1)
    D[i, j] = (-1.0) ** (i + j) / (z[i] - z[j])
    D[:, 0] *= 0.5
    D[n - 1, :] *= 2.0
    iu, ju = np.triu_indices(n, 1)
    D[iu, ju] = -D[n - 1 - iu, n - 1 - ju]
    np.fill_diagonal(D, 0.0)
    np.fill_diagonal(D, -D.sum(axis=1))
    if mapping == 1:
        t = np.tan(np.pi / 2 * z)
        zc = 2 / np.pi * np.arctan(coef * t)
        D = np.diag(1 / coef * (1 + (coef * t) ** 2) / (1 + t ** 2)) @ D
    elif mapping == 2:
        zc = np.arcsin(coef * z) / np.arcsin(coef)
        D = np.diag(1 / coef * np.cos(np.arcsin(coef * z)) * np.arcsin(coef)) @ D
    elif mapping == 3:
        t = np.tan(np.pi / 4 * (z - 1))
        zc = 4 / np.pi * np.arctan(coef * t) + 1
        D = np.diag(1 / coef * (1 + (coef * t) ** 2) / (1 + t ** 2)) @ D
    if mapping != 0:
        grid.gridlenz = grid._gridlenz(zc)
    D2 = D @ D
    np.fill_diagonal(D2, 0.0)
    np.fill_diagonal(D2, -D2.sum(axis=1))
    return D, D2


# ----------------------------------------------------------------------------
# Pruned plane transforms (RealCplxCube::DftForward / DftBackward)
# ----------------------------------------------------------------------------
def dft_forward(g: Grid, phys: np.ndarray) -> np.ndarray:
    """(.., Nz, Ny, Nx) real -> (.., Nxh, Nyc, Nz) complex; x r2c, y c2c, /(NxNy).

    src/cube_real_cplx.cc:525-539 ('ffn': no z transform), pruning per
    build/ftran.F90:122-248 (keep kx 0..Nxc/2; ky 0..Nyc/2-1 and Ny-Nyc/2..Ny-1).
    """
    F = sfft.rfft(phys, axis=-1, workers=WORKERS)[..., :g.nxh]
    F = sfft.fft(F, axis=-2, workers=WORKERS)[..., g.yidx, :]
    F *= 1.0 / (g.nx * g.ny)
    return np.ascontiguousarray(np.swapaxes(F, -1, -3))


def dft_backward(g: Grid, spec: np.ndarray) -> np.ndarray:
    """(.., Nxh, Nyc, Nz) complex -> (.., Nz, Ny, Nx) real; zero-fill, unscaled.

    src/cube_real_cplx.cc:542-555, build/btran.F90:137-243.  The x c2r ignores
    the imaginary part of the kx=0 (and Nyquist) coefficient, as FFTW does.
    """
    S = np.swapaxes(spec, -1, -3)
    full = np.zeros(S.shape[:-2] + (g.ny, g.nx // 2 + 1), dtype=np.complex128)
    full[..., g.yidx, :g.nxh] = S
    full = sfft.ifft(full, axis=-2, norm="forward", workers=WORKERS)
    return sfft.irfft(full, n=g.nx, axis=-1, norm="forward", workers=WORKERS)


def zmul(A: np.ndarray, X: np.ndarray) -> np.ndarray:
    """Real Nz x Nz operator applied along z: R = A * X (src/cube_real_cplx.cc:461-471).

    X is (.., Nxh, Nyc, Nz) complex (or (.., M, Nz)); the product is done as a real
    GEMM on stacked real/imaginary parts.
    """
    R = np.stack([X.real, X.imag])
    Y = R @ A.T
    return Y[0] + 1j * Y[1]


def zrow(vec: np.ndarray, X: np.ndarray) -> np.ndarray:
    """Row functional along z: vec . X[..., :]  (Multiply(cmat,int), cube_real_cplx.cc:480-486)."""
    return X.real @ vec + 1j * (X.imag @ vec)


# ----------------------------------------------------------------------------
# Helmholtz decomposition: CmDz2DecompositionCplx (src/cmdz2_decomposition.cc)
# ----------------------------------------------------------------------------
class Dz2Decomposition:
    def __init__(self, g: Grid, D1: np.ndarray, D2: np.ndarray, bc, stepcoef,
                 eig_override=None):
        n = g.nz
        A = D2.copy()                                  # :47-50
        A[0] = bc[1] * D1[0]
        A[n - 1] = bc[3] * D1[n - 1]
        A[0, 0] += bc[0]
        A[n - 1, n - 1] += bc[2]
        a11, ann, a1n, an1 = A[0, 0], A[n - 1, n - 1], A[0, n - 1], A[n - 1, 0]
        den = 1.0 / (an1 * a1n - a11 * ann)            # :54-58
        fbb = np.zeros(n); ftb = np.zeros(n); fbf = np.zeros(n); ftf = np.zeros(n)
        s = slice(1, n - 1)                            # :71-83
        fbb[s] = (ann * A[0, s] - a1n * A[n - 1, s]) * den
        ftb[s] = (a11 * A[n - 1, s] - an1 * A[0, s]) * den
        fbf[s] = (ann * A[s, 0] - an1 * A[s, n - 1]) * den
        ftf[s] = (a11 * A[s, n - 1] - a1n * A[s, 0]) * den
        fbb[0] = -ann * den; fbb[n - 1] = a1n * den
        ftb[0] = an1 * den; ftb[n - 1] = -a11 * den
        # condensed interior operator: :88-96
        F = A[s, s] + np.outer(A[s, 0], fbb[s]) + np.outer(A[s, n - 1], ftb[s])
        if eig_override is None:
            lam, V = np.linalg.eig(F)                  # eig_gen, :99-101
        else:
            lam, V = eig_override(F)
        E = np.zeros((n, n)); E[s, s] = V.real; E[0, 0] = E[n - 1, n - 1] = 1.0
        Ei = np.zeros((n, n)); Ei[s, s] = np.linalg.inv(V.real)
        Ei[0, 0] = Ei[n - 1, n - 1] = 1.0
        self.n = n
        self.bc = list(bc)
        self.A = A
        self.F = F
        self.fbb, self.ftb, self.fbf, self.ftf = fbb, ftb, fbf, ftf
        self.E, self.Einv = E, Ei
        self.lam = np.zeros(n)
        self.lam[s] = lam.real                         # imag part zeroed, :100
        self.assemble(g, stepcoef)

    def assemble(self, g: Grid, stepcoef):
        """Per-stage reciprocal R_s[m, z] (src/cmdz2_decomposition.cc:234-297)."""
        n = self.n
        self.stepcoef = list(stepcoef)
        self.R = []
        for sv in stepcoef:
            R = np.ones((g.M, n))
            R[:, 1:n - 1] = 1.0 / ((g.dx2 + g.dy2)[:, None] + self.lam[None, 1:n - 1] + sv)
            if abs(sv) < COMPARE_NUMBER_SMALL:         # single rank always holds the mean mode
                for k in range(1, n - 1):
                    if abs(self.lam[k]) < COMPARE_NUMBER_SMALL:
                        R[0, k] = 0.0
            self.R.append(R)

    def solve(self, target: np.ndarray, stage: int, forward_fix: bool) -> np.ndarray:
        """E*(R_s .* (E^-1 * t)) plus the boundary rows.

        forward_fix=True: interior rows += fbf*row0 + ftf*row(N-1) first
        (phase_carrier_flat.cc:877-881, phase_scalar_flat.cc:649-653);
        forward_fix=False: rows 0 and N-1 of the target are zeroed (pressure,
        phase_carrier_flat.cc:966-967).  Row 0 := fbb.y, then row N-1 := ftb.y
        using the already replaced row 0 (phase_carrier_flat.cc:885-887).
        The target is modified in place as in the reference.
        """
        n = self.n
        t = target
        if forward_fix:
            t[..., 1:n - 1] += self.fbf[1:n - 1] * t[..., :1] + self.ftf[1:n - 1] * t[..., n - 1:]
        else:
            t[..., 0] = 0.0
            t[..., n - 1] = 0.0
        Rs = self.R[stage]
        y = zmul(self.E, Rs.reshape(t.shape) * zmul(self.Einv, t))
        y[..., 0] = zrow(self.fbb, y)
        y[..., n - 1] = zrow(self.ftb, y)
        return y


# ----------------------------------------------------------------------------
# Restart files: "IOControlLevelOne\n" then Armadillo binary complex cubes
# ("ARMA_CUB_BIN_FC016\n<nz> <nyc> <nxh*dim>\n" + column-major doubles).
# src/variable_carrier_flat.cc:143-377, src/variable_scalar_flat.cc
# ----------------------------------------------------------------------------
def write_arma_cplx(f, spec: np.ndarray):
    """spec (dim, Nxh, Nyc, Nz) -> ccube(Nz, Nyc, Nxh*dim) binary."""
    dim, nxh, nyc, nz = spec.shape
    f.write(b"ARMA_CUB_BIN_FC016\n")
    f.write(f"{nz} {nyc} {nxh * dim}\n".encode())
    f.write(np.ascontiguousarray(spec, dtype=np.complex128).tobytes())


def read_arma_cplx(f, dim: int) -> np.ndarray:
    head = f.readline().strip()
    if head != b"ARMA_CUB_BIN_FC016":
        raise ValueError(f"not an Armadillo complex cube: {head!r}")
    nz, nyc, nslice = (int(v) for v in f.readline().split())
    data = np.frombuffer(f.read(16 * nz * nyc * nslice), dtype=np.complex128)
    return data.reshape(dim, nslice // dim, nyc, nz).copy()


def write_phase_file(path: str, fields: List[np.ndarray]):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "wb") as f:
        f.write(b"IOControlLevelOne\n")
        for a in fields:
            write_arma_cplx(f, a)


def read_phase_file(path: str, dims: List[int]) -> List[np.ndarray]:
    with open(path, "rb") as f:
        level = f.readline().strip()
        if level != b"IOControlLevelOne":
            raise ValueError("Variable::Load > Wrong Request of IO Level One!")
        return [read_arma_cplx(f, d) for d in dims]


# ----------------------------------------------------------------------------
# Analytic laminar solution (tmtools/get_loflow.m:17-20) and synthetic states
# ----------------------------------------------------------------------------
def stokes_profile(re: float, z: np.ndarray, t: float, free_slip_top: bool = False) -> np.ndarray:
    """Oscillatory laminar profile u(z,t) for du/dt = cos t + u_zz/Re.

    No-slip at both walls: Re{i(cosh(k z)/cosh(k) - 1) e^{it}}, k = (1+i)/sqrt(2) sqrt(Re)
    (tmtools/get_loflow.m).  With a free-slip top the homogeneous part is
    cosh(k(z-1))/cosh(2k), which satisfies u'(1) = 0 and u(-1) = 0.
    """
    k = (1 + 1j) / np.sqrt(2) * np.sqrt(re)
    if free_slip_top:
        prof = 1j * (np.cosh(k * (z - 1)) / np.cosh(2 * k) - 1)
    else:
        prof = 1j * (np.cosh(k * z) / np.cosh(k) - 1)
    return np.real(prof * np.exp(1j * t))


def make_initial_state(cfg: CaseConfig, seed: int = 0, noise: float = 1e-4,
                       scalar_noise: float = 0.1, modes: int = 3, scalar_mean=1.0):
    """Seeded synthetic restart state (spectral uvw (3,..), p (1,..), phi (1,..)).

    Mean mode: the analytic laminar profile at t = 0.  Perturbation: the curl of a
    seeded vector potential with wall-vanishing envelope (1 - z^2)^2 and Fourier
    modes |kx|,|ky| <= `modes`, scaled so that its peak equals `noise`.  phi is
    `scalar_mean` + `scalar_noise` * uniform(-1, 1) noise, mean mode set to
    `scalar_mean` (a number, or one value per z plane).
    """
    g = Grid(cfg)
    rng = np.random.default_rng(seed)
    z = g.gridz
    X, Y = np.meshgrid(g.gridx, g.gridy, indexing="xy")      # (ny, nx)
    env = (1 - z ** 2) ** 2
    denv = -4 * z * (1 - z ** 2)
    kx1 = 2 * np.pi / cfg.lx
    ky1 = 2 * np.pi / cfg.ly
    psi = np.zeros((3, g.nz, g.ny, g.nx))
    dpsi_dx = np.zeros_like(psi); dpsi_dy = np.zeros_like(psi); dpsi_dz = np.zeros_like(psi)
    mx = min(modes, g.nxc // 2)
    my = min(modes, g.nyc // 2 - 1) if g.nyc >= 4 else 0
    for c in range(3):
        for a in range(0, mx + 1):
            for b in range(-my, my + 1):
                if a == 0 and b == 0:
                    continue
                amp = rng.standard_normal(2)
                ph = a * kx1 * X + b * ky1 * Y
                f = amp[0] * np.cos(ph) + amp[1] * np.sin(ph)
                fx = a * kx1 * (-amp[0] * np.sin(ph) + amp[1] * np.cos(ph))
                fy = b * ky1 * (-amp[0] * np.sin(ph) + amp[1] * np.cos(ph))
                psi[c] += env[:, None, None] * f
                dpsi_dx[c] += env[:, None, None] * fx
                dpsi_dy[c] += env[:, None, None] * fy
                dpsi_dz[c] += denv[:, None, None] * f
    up = np.stack([dpsi_dy[2] - dpsi_dz[1], dpsi_dz[0] - dpsi_dx[2], dpsi_dx[1] - dpsi_dy[0]])
    peak = np.abs(up).max()
    if peak > 0:
        up *= noise / peak
    opentop = abs(cfg.bc_u[2]) <= COMPARE_NUMBER_SMALL and abs(cfg.bc_u[3] - 1) <= COMPARE_NUMBER_SMALL
    uvw = dft_forward(g, up)
    prof = stokes_profile(cfg.reynolds, z, 0.0, free_slip_top=opentop)
    prof[0] = 0.0
    if not opentop:
        prof[-1] = 0.0
    uvw[0, 0, 0, :] += prof
    p = np.zeros((1, g.nxh, g.nyc, g.nz), dtype=np.complex128)
    mean = np.broadcast_to(np.asarray(scalar_mean, dtype=np.float64), (g.nz,))
    phi_phys = mean[None, :, None, None] + scalar_noise * rng.uniform(-1.0, 1.0, size=(1, g.nz, g.ny, g.nx))
    phi = dft_forward(g, phi_phys)
    phi[0, 0, 0, :] = mean
    return uvw, p, phi


# ----------------------------------------------------------------------------
# The solver: FlatChannelSolver's configure + step loop with both phases
# ----------------------------------------------------------------------------
class OracleSolver:
    """FP64 restatement of FlatChannelSolver::{Configure,Execute} for one case."""

    def __init__(self, cfg: CaseConfig, uvw: np.ndarray, p: np.ndarray,
                 phi: Optional[np.ndarray] = None, eig_override=None):
        self.cfg = cfg
        g = self.g = Grid(cfg)
        self.D1, self.D2 = chebyshev_d1_d2(g, cfg.mapping, cfg.mapping_coef)
        n = g.nz
        # --- TimeStepper::Configure (src/stepper_time.cc:215-246)
        self.output_time_index = 0
        if cfg.output_based_on_step:
            self.step = max(0, cfg.startstep)
            self.dt = cfg.dt
            self.time = self.step * self.dt
            self.isforward = self.step <= cfg.maxstep
        else:
            self.step = 0
            self.dt = cfg.initial_time_step
            self.time = cfg.start_time_index * cfg.output_interval if cfg.start_time_index > 0 else 0.0
            self.output_time_index = cfg.start_time_index
            self.isforward = self.time <= cfg.max_marching_time
        self.isoutput = False
        self.cfl = 0.0
        self.alternation = False
        # --- FlatCarrierPhase::Configure (src/phase_carrier_flat.cc:178-246)
        sc = [-cfg.reynolds / self.dt / RK3[2, s] for s in range(3)]
        self.dec_u = Dz2Decomposition(g, self.D1, self.D2, cfg.bc_u, sc, eig_override)
        self.dec_v = Dz2Decomposition(g, self.D1, self.D2, cfg.bc_v, sc, eig_override)
        self.dec_w = Dz2Decomposition(g, self.D1, self.D2, cfg.bc_w, sc, eig_override)
        self.dec_p = Dz2Decomposition(g, self.D1, self.D2, cfg.bc_p, [0.0, 0.0, 0.0], eig_override)
        shp = (g.nxh, g.nyc, n)
        self.uvw = np.array(uvw, dtype=np.complex128).reshape((3,) + shp)
        self.p = np.array(p, dtype=np.complex128).reshape((1,) + shp)
        # FlatCarrierVariable::Configure (variable_carrier_flat.cc:386-421)
        self.dpdxyz = self.gradient(self.p[0])
        self.huvw = np.zeros_like(self.uvw)
        self.dudxyz = np.zeros((3, 3) + shp, dtype=np.complex128)   # dudxyz/dvdxyz/dwdxyz[0]
        self.dudxyz_phys = None
        self.dudxyztmp = np.zeros((3,) + shp, dtype=np.complex128)
        # FlatCarrierBoundary (boundary_carrier_flat.cc:25-48, 255-269)
        z3 = np.zeros((3, g.nxh, g.nyc), dtype=np.complex128)
        self.dp1m1top = z3.copy(); self.dp1m1bot = z3.copy()
        self.dp2m1top = z3.copy(); self.dp2m1bot = z3.copy()
        self.dp1m2top = z3.copy(); self.dp1m2bot = z3.copy()
        self.dp2m2top = z3.copy(); self.dp2m2bot = z3.copy()
        self.olddt = self.dt
        bu = cfg.bc_u                                   # boundary.cc:59-71
        self.opentop = abs(bu[2] - 0) <= COMPARE_NUMBER_SMALL and abs(bu[3] - 1) <= COMPARE_NUMBER_SMALL
        self.uvwnl = dft_backward(g, self.uvw)
        self.flocal = np.zeros(50)
        self.fglobal = np.zeros(50)
        self.bulkvelocity = 1.0
        # --- FlatScalarPhase::Configure (src/phase_scalar_flat.cc:176-221)
        self.scalar = cfg.nphase > 1
        if self.scalar:
            scs = [-cfg.reynolds * cfg.schmidt / self.dt / RK3[2, s] for s in range(3)]
            rsw = cfg.reynolds * cfg.schmidt * cfg.settling
            bcs = [rsw * BOUNDARY_COEF_SCALE, BOUNDARY_COEF_SCALE, rsw * BOUNDARY_COEF_SCALE, BOUNDARY_COEF_SCALE]
            self.dec_s = Dz2Decomposition(g, self.D1, self.D2, bcs, scs, eig_override)
            self.phi = np.array(phi, dtype=np.complex128).reshape((1,) + shp)
            self.hphi = np.zeros_like(self.phi)
            self.uvw_s = np.zeros_like(self.uvw)
            self.uvwnl_s = dft_backward(g, self.uvw_s)
            self.features_scalar_flux = (0.0, 0.0)

    # -- SpaceStepper operators (src/stepper_space.cc:373-408)
    def gradient(self, f):
        g = self.g
        fm = f.reshape(g.M, g.nz)
        out = np.empty((3, g.M, g.nz), dtype=np.complex128)
        out[0] = g.dx1[:, None] * fm
        out[1] = g.dy1[:, None] * fm
        out[2] = zmul(self.D1, fm)
        return out.reshape((3,) + f.shape)

    def gradient_tmp(self, t3):
        g = self.g
        t = t3.reshape(3, g.M, g.nz)
        out = np.empty((3, g.M, g.nz), dtype=np.complex128)
        out[0] = g.dx1[:, None] * t[0]
        out[1] = g.dy1[:, None] * t[1]
        out[2] = zmul(self.D1, t[2])
        return out.reshape(t3.shape)

    def laplacian_like(self, f):
        """D2*f + cmdx2 % f + cmdy2 % f (phase_carrier_flat.cc:517-528)."""
        g = self.g
        fm = f.reshape(g.M, g.nz)
        return (zmul(self.D2, fm) + (g.dx2[:, None] * fm + g.dy2[:, None] * fm)).reshape(f.shape)

    def mean_col(self, a):
        """cmat column 0 (kx=ky=0) of a spectral component: shape (Nz,)."""
        return a[0, 0, :]

    # -- FlatCarrierPhase::NonlinearVelocity (src/phase_carrier_flat.cc:716-813)
    def nonlinear_velocity(self):
        g = self.g
        un = self.uvwnl
        if self.alternation:
            prods = np.empty((3, 3) + un.shape[1:])
            for i in range(3):
                for j in range(3):
                    prods[i, j] = un[i] * un[j]
            P = dft_forward(g, prods.reshape((9,) + un.shape[1:])).reshape((3, 3, g.nxh, g.nyc, g.nz))
            adv = np.empty_like(self.uvw)
            for i in range(3):
                gt = self.gradient_tmp(P[i])
                adv[i] = gt[0] + gt[1] + gt[2]
            for i in range(3):
                self.dudxyz[i] = self.gradient(self.uvw[i])
            if self.scalar:
                self.dudxyz_phys = dft_backward(g, self.dudxyz.reshape((9,) + self.uvw.shape[1:])).reshape(
                    (3, 3) + un.shape[1:])
            return adv
        for i in range(3):
            self.dudxyz[i] = self.gradient(self.uvw[i])
        self.dudxyz_phys = dft_backward(g, self.dudxyz.reshape((9,) + self.uvw.shape[1:])).reshape(
            (3, 3) + un.shape[1:])
        dp = self.dudxyz_phys
        advr = np.empty_like(un)
        for i in range(3):
            advr[i] = un[0] * dp[i, 0] + un[1] * dp[i, 1] + un[2] * dp[i, 2]
        return dft_forward(g, advr)

    def _force(self):
        """Mean-mode driving force (src/phase_carrier_flat.cc:365-501)."""
        cfg = self.cfg
        dt, t = self.dt, self.time
        tt = t - dt / 2 if cfg.output_based_on_step else t + dt / 2
        f1 = f2 = 0.0
        ft = cfg.force_type
        fd, fa = cfg.force_direction, cfg.force_amplitude
        if ft == 1:
            if fd[0] == 1: f1 = fa[0]
            elif fd[0] == 2: f2 = fa[0]
        elif ft == 2:
            a = fa[1]
            if fd[1] == 1: f1 = a * np.cos(a * tt)
            elif fd[1] == 2: f2 = a * np.cos(a * tt)
        elif ft == 3:
            if fd[0] == 1: f1 = fa[0]
            elif fd[0] == 2: f2 = fa[0]
            a = fa[1]
            if fd[1] == 1: f1 += a * np.cos(a * tt)
            elif fd[1] == 2: f2 += a * np.cos(a * tt)
        elif ft == 4:
            if fd[0] == 1: f1 = fa[0]
            elif fd[0] == 2: f2 = fa[0]
            a = fa[1]
            T, t0, lastp, tarp = fa[0], fa[1], fa[2], fa[3]
            damp = -np.log(tarp) / (lastp + 0.25) / T
            val = (a * np.cos(a * tt) - damp * np.sin(a * tt)) * np.exp(-damp * (t - t0))
            if fd[1] == 1: f1 += val
            elif fd[1] == 2: f2 += val
        return f1, f2

    def boundary_apply(self, stage, rhs):
        """FlatCarrierBoundary::Apply (src/boundary_carrier_flat.cc:185-246)."""
        dt = self.dt
        c3m0 = RK3[2, stage]; c3m1 = RK3[2, (stage + 2) % 3]; c3m2 = RK3[2, (stage + 1) % 3]
        if stage == 0:
            xm0, xm1, xm2 = 2 * c3m0 * dt, 0.0, 2 * (0 - c3m1) * self.olddt
        elif stage == 1:
            xm0, xm1, xm2 = 2 * (c3m0 + c3m1) * dt, 2 * c3m1 * dt, 0.0
        else:
            xm0, xm1, xm2 = 2 * (c3m0 + c3m1 + c3m2) * dt, 2 * (c3m1 + c3m2) * dt, 2 * c3m2 * dt
        r = (xm0 - xm1) / (xm1 - xm2)
        fac = 2 * dt * c3m0
        rhs[..., -1] = fac * ((1 + r) * self.dp1m1top + (0 - r) * self.dp1m2top)
        rhs[..., 0] = fac * ((1 + r) * self.dp1m1bot + (0 - r) * self.dp1m2bot)
        if self.opentop:
            rhs[0, ..., -1] = fac * ((1 + r) * self.dp2m1top[0] + (0 - r) * self.dp2m2top[0])
            rhs[1, ..., -1] = fac * ((1 + r) * self.dp2m1top[1] + (0 - r) * self.dp2m2top[1])

    # -- FlatCarrierPhase::Predict (src/phase_carrier_flat.cc:272-559)
    def carrier_predict(self, stage):
        cfg, g = self.cfg, self.g
        dt = self.dt
        c1, c2, c3 = RK3[0, stage], RK3[1, stage], RK3[2, stage]
        adv = self.nonlinear_velocity()
        self.huvw = c1 * self.huvw - dt * adv
        if self.scalar and cfg.affected_by_scalar:
            coef = dt * cfg.averaged_concentration / cfg.froude ** 2 * (cfg.specific_gravity - 1)
            ph = self.phi[0]
            if cfg.slope_direction == 1:
                self.huvw[0] = self.huvw[0] + coef * ph * np.sin(cfg.slope)
            elif cfg.slope_direction == 2:
                self.huvw[1] = self.huvw[1] + coef * ph * np.sin(cfg.slope)
            self.huvw[2] = self.huvw[2] - coef * ph * np.cos(cfg.slope)
        f1, f2 = self._force()
        self.huvw[0, 0, 0, :] += dt * f1
        self.huvw[1, 0, 0, :] += dt * f2
        self.bulkvelocity = np.trapezoid(self.uvw[0, 0, 0, :].real, g.gridz) / 2
        lap = np.stack([self.laplacian_like(self.uvw[i]) for i in range(3)])
        redtc3 = -cfg.reynolds / dt / c3
        rhs = redtc3 * c2 * self.huvw + redtc3 * self.uvw - lap
        self.boundary_apply(stage, rhs)
        rhs[0, 0, 0, -1] = cfg.bc_u[4]
        rhs[1, 0, 0, -1] = cfg.bc_v[4]
        rhs[2, 0, 0, -1] = cfg.bc_w[4]
        self.suvw = np.stack([
            self.dec_u.solve(rhs[0].reshape(g.M, g.nz), stage, True).reshape(rhs.shape[1:]),
            self.dec_v.solve(rhs[1].reshape(g.M, g.nz), stage, True).reshape(rhs.shape[1:]),
            self.dec_w.solve(rhs[2].reshape(g.M, g.nz), stage, True).reshape(rhs.shape[1:])])

    # -- FlatCarrierPhase::Correct (src/phase_carrier_flat.cc:566-709)
    def carrier_correct(self, stage):
        cfg, g = self.cfg, self.g
        dt = self.dt
        c3 = RK3[2, stage]
        s = self.suvw.reshape(3, g.M, g.nz)
        divs = zmul(self.D1, s[2]) + g.dx1[:, None] * s[0] + g.dy1[:, None] * s[1]
        rhsp = 0.5 / dt / c3 * divs
        self.p[0] = self.dec_p.solve(rhsp, stage, False).reshape(self.p.shape[1:])
        self.dpdxyz = self.gradient(self.p[0])
        if self.opentop:
            self.dudxyztmp = self.gradient(self.dpdxyz[2])
        # FlatCarrierBoundary::Update (boundary_carrier_flat.cc:131-170)
        if stage == 2:
            self.olddt = dt
        self.dp1m2top = self.dp1m1top; self.dp2m2top = self.dp2m1top
        self.dp1m2bot = self.dp1m1bot; self.dp2m2bot = self.dp2m1bot
        self.dp1m1bot = self.dpdxyz[..., 0].copy()
        self.dp1m1top = self.dpdxyz[..., -1].copy()
        if self.opentop:
            self.dp2m1bot = self.dudxyztmp[..., 0].copy()
            self.dp2m1top = self.dudxyztmp[..., -1].copy()
        self.uvw = self.suvw - 2 * dt * c3 * self.dpdxyz
        self.uvw[2, 0, 0, :] = 0.0
        self.uvwnl = dft_backward(g, self.uvw)
        if stage == 2:
            self._features()

    def _features(self):
        """Stage-2 features (src/phase_carrier_flat.cc:633-703); single rank."""
        g = self.g
        un = self.uvwnl
        fl = self.flocal
        for i in range(3):
            fl[i] = np.abs(un[i]).max()
            fl[3 + i] = np.abs(un[i][0]).max()
            fl[6 + i] = np.abs(un[i][-1]).max()
        maxulen = (np.abs(un[0]) / g.lengthminx + np.abs(un[1]) / g.lengthminy
                   + np.abs(un[2]) / g.gridlenz[:, None, None])
        fl[19] = maxulen.max()
        fg = np.zeros(50)
        fg[:] = fl
        for k, (i, row) in enumerate([(0, 0), (1, 0), (2, 0), (0, -1), (1, -1), (2, -1)]):
            fg[10 + k] = self.dudxyz[i, 2, 0, 0, row].real
        for k in (21, 22, 23, 24, 25, 28, 29):
            fg[k] = fl[k]
        self.fglobal = fg

    # -- FlatScalarPhase::Predict (src/phase_scalar_flat.cc:245-284)
    def scalar_predict(self, stage):
        cfg, g = self.cfg, self.g
        self.uvw_s = self.uvw.copy()
        ws = cfg.settling
        if cfg.slope_direction == 1:
            self.uvw_s[0, 0, 0, :] += ws * np.sin(cfg.slope)
        elif cfg.slope_direction == 2:
            self.uvw_s[1, 0, 0, :] += ws * np.sin(cfg.slope)
        self.uvw_s[2, 0, 0, :] -= ws * np.cos(cfg.slope)
        self.uvwnl_s = dft_backward(g, self.uvw_s)

    def nonlinear_scalar(self):
        """FlatScalarPhase::NonlinearPressure (src/phase_scalar_flat.cc:552-599)."""
        g = self.g
        un = self.uvwnl_s
        if self.alternation:
            pp = dft_backward(g, self.phi)[0]
            P = dft_forward(g, pp[None] * un)
            gt = self.gradient_tmp(P)
            return (gt[0] + gt[1] + gt[2])[None]
        gp = dft_backward(g, self.gradient(self.phi[0]))
        advr = un[0] * gp[0] + un[1] * gp[1] + un[2] * gp[2]
        return dft_forward(g, advr[None])

    # -- FlatScalarPhase::Correct (src/phase_scalar_flat.cc:291-533)
    def scalar_correct(self, stage):
        cfg, g = self.cfg, self.g
        dt = self.dt
        c1, c2, c3 = RK3[0, stage], RK3[1, stage], RK3[2, stage]
        adv = self.nonlinear_scalar()
        self.hphi = c1 * self.hphi - dt * adv
        lap = self.laplacian_like(self.phi[0])[None]
        redtc3 = -cfg.reynolds * cfg.schmidt / dt / c3
        rhs = redtc3 * c2 * self.hphi + redtc3 * self.phi - lap
        rhs[..., 0] = 0.0                               # boundary_scalar_flat.cc:144-156
        rhs[..., -1] = 0.0
        if cfg.scalar_bc == 1:
            tauc, susp = cfg.critical_shear, cfg.erosion_rate
            dp = self.dudxyz_phys
            tau = np.sqrt(dp[0, 2] * dp[0, 2] + dp[1, 2] * dp[1, 2]) / cfg.reynolds
            tau = np.where(tau < tauc, 0.0, susp * (tau / tauc - 1)) if tauc != 0 else \
                np.where(tau < tauc, 0.0, susp * (tau / tauc - 1))
            ero = dft_forward(g, tau[None])
            wsc = cfg.settling * np.cos(cfg.slope)
            row = ero[0, ..., 0] - wsc * self.phi[0, ..., 0] * cfg.averaged_concentration
            rhs[0, ..., 0] = -1 * row * cfg.reynolds * cfg.schmidt / cfg.averaged_concentration * BOUNDARY_COEF_SCALE
            self.flocal[28] = ero[0, 0, 0, 0].real
            self.flocal[29] = (wsc * self.phi[0, 0, 0, 0] * cfg.averaged_concentration).real
        phi = self.dec_s.solve(rhs[0].reshape(g.M, g.nz), stage, True)
        phi = phi.reshape((1,) + self.phi.shape[1:])
        self.phi = self.positivity_filter(phi)
        self.flocal[21] = np.trapezoid(self.phi[0, 0, 0, :].real, g.gridz) / 2
        if stage == 2 and cfg.slope_direction > 0:
            self.flocal[22] = np.trapezoid(self.uvw_s[0, 0, 0, :].real, g.gridz) / 2
            self.flocal[24] = np.trapezoid(self.uvw_s[1, 0, 0, :].real, g.gridz) / 2
            self.flocal[23] = 0.0
            self.flocal[25] = 0.0
            if self.step % 10 == 0:
                pp = self._phi_phys
                f0 = dft_forward(g, (self.uvwnl_s[0] * pp)[None])
                self.flocal[23] = np.trapezoid(f0[0, 0, 0, :].real, g.gridz) / 2
                f1 = dft_forward(g, (self.uvwnl_s[1] * pp)[None])
                self.flocal[25] = np.trapezoid(f1[0, 0, 0, :].real, g.gridz) / 2

    def positivity_filter(self, phi):
        """Bartnicki filter, 5 sweeps of per-z-plane sums (phase_scalar_flat.cc:419-478)."""
        g = self.g
        pp = dft_backward(g, phi)[0]
        for _ in range(5):
            pos = pp > 0
            neg = pp < 0
            sp = np.where(pos, pp, 0.0).sum(axis=(1, 2))
            cp = pos.sum(axis=(1, 2)).astype(np.float64)
            sn = np.where(neg, pp, 0.0).sum(axis=(1, 2))
            sz = np.where(~pos & ~neg, pp, 0.0).sum(axis=(1, 2))
            kill = (sp + sz + sn) < 0
            with np.errstate(divide="ignore", invalid="ignore"):
                add = np.where(cp > 0, sn / np.where(cp > 0, cp, 1.0), 0.0)
            pp = np.where(pos, pp + add[:, None, None], 0.0)
            pp[kill] = 0.0
        self._phi_phys = pp
        return dft_forward(g, pp[None])

    # -- FlatChannelSolver::Execute, one pass of the while loop (solver_channel_flat.cc:199-293)
    def time_update(self):
        """TimeStepper::Update (src/stepper_time.cc:72-113)."""
        cfg = self.cfg
        if not self.isforward:
            return
        maxulen = self.fglobal[19]
        self.step += 1
        self.time = self.time + self.dt
        self.isforward = self.step < cfg.maxstep
        self.isoutput = self.step % cfg.writeinterval == 0
        self.cfl = maxulen * self.dt
        if self.cfl > cfg.maxcfl:
            self.isforward = False
            self.isoutput = True

    def time_update2(self):
        """TimeStepper::Update2 (src/stepper_time.cc:117-208): the adaptive-dt
        branch.  time advances by the previous dt, then dt is rescaled towards
        the CFL band and clipped to land on the next output time."""
        cfg = self.cfg
        if not self.isforward:
            return
        maxulen = self.fglobal[19]
        self.step += 1
        self.time = self.time + self.dt
        self.isforward = self.time < cfg.max_marching_time
        self.cfl = maxulen * self.dt
        if self.cfl > 0:
            top, bot = cfg.cfl_adjust_scale[0], cfg.cfl_adjust_scale[1]
            if self.cfl > top * cfg.maxcfl:
                self.dt = self.dt * top
                while maxulen * self.dt > top * cfg.maxcfl:
                    self.dt = self.dt * top
            elif self.cfl < bot * cfg.maxcfl:
                self.dt = self.dt * 1.05
            if (self.time + self.dt) / cfg.output_interval - self.output_time_index - 1 >= 0:
                dttmp = (self.output_time_index + 1) * cfg.output_interval - self.time
                if dttmp < cfg.initial_time_step / 100:
                    self.dt = self.dt / 20
                else:
                    self.dt = dttmp
                self.output_time_index += 1
                self.isoutput = True
            else:
                self.isoutput = False
        if self.cfl > cfg.maxcfl * 1.1 or self.dt < cfg.initial_time_step / 1000:
            self.isforward = False
            self.isoutput = True

    def phase_update(self):
        """FlatCarrierPhase::Update / FlatScalarPhase::Update
        (src/phase_carrier_flat.cc:248-262, src/phase_scalar_flat.cc:225-238):
        the reciprocals re-assembled for the current dt (pressure unchanged)."""
        cfg, g = self.cfg, self.g
        sc = [-cfg.reynolds / self.dt / RK3[2, s] for s in range(3)]
        for d in (self.dec_u, self.dec_v, self.dec_w):
            d.assemble(g, sc)
        if self.scalar:
            self.dec_s.assemble(g, [-cfg.reynolds * cfg.schmidt / self.dt / RK3[2, s] for s in range(3)])

    def run_step(self):
        if self.cfg.output_based_on_step:
            self.time_update()
        else:
            self.time_update2()
            self.phase_update()
        for stage in range(3):
            self.carrier_predict(stage)
            self.carrier_correct(stage)
            if self.scalar:
                self.scalar_predict(stage)
                self.scalar_correct(stage)
        self.alternation = not self.alternation

    def state(self) -> Dict[str, np.ndarray]:
        out = {"u": self.uvw[0].copy(), "v": self.uvw[1].copy(), "w": self.uvw[2].copy(),
               "p": self.p[0].copy()}
        if self.scalar:
            out["c"] = self.phi[0].copy()
        return out


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


# ----------------------------------------------------------------------------
# Post-processor: swirling strength (src/postprocessor_channel_flat.cc:195-236)
# ----------------------------------------------------------------------------
def swirling_strength(cfg: CaseConfig, uvw: np.ndarray) -> np.ndarray:
    """lambda_ci per physical point: the largest |imaginary part| of the
    eigenvalues (eig_gen) of the velocity-gradient tensor A(i, j) = du_i/dx_j,
    the gradients taken as SpaceStepper::Gradient does (i kx, i ky, D1) and
    transformed back.  uvw: (3, Nxh, Nyc, Nz) spectral; returns (Nz, Ny, Nx)."""
    g = Grid(cfg)
    D1, _ = chebyshev_d1_d2(g, cfg.mapping, cfg.mapping_coef)
    u = np.asarray(uvw, dtype=np.complex128).reshape(3, g.nxh, g.nyc, g.nz)
    grads = np.empty((3, 3) + u.shape[1:], dtype=np.complex128)
    for i in range(3):
        fm = u[i].reshape(g.M, g.nz)
        grads[i, 0] = (g.dx1[:, None] * fm).reshape(u.shape[1:])
        grads[i, 1] = (g.dy1[:, None] * fm).reshape(u.shape[1:])
        grads[i, 2] = zmul(D1, fm).reshape(u.shape[1:])
    phys = dft_backward(g, grads.reshape((9,) + u.shape[1:]))        # (9, Nz, Ny, Nx)
    A = np.moveaxis(phys.reshape(3, 3, -1), -1, 0)                   # (points, 3, 3)
    ev = np.linalg.eigvals(A)
    return np.abs(ev.imag).max(axis=1).reshape(g.nz, g.ny, g.nx)
