"""Host-side wrapper of one GPU case (tg_ctx) mirroring the reference plugins.

`ChannelCase` exposes the plugin methods of the reference -- the phases'
Predict/Correct (src/phase.h:25-114), the time loop of
FlatChannelSolver::Execute (src/solver_channel_flat.cc:199-293), restart
Load/Save -- on top of the C ABI.  State arrays crossing the boundary use the
reference's restart layout: complex (dim, Nxh, Nyc, Nz), z fastest.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

from . import _lib
from ._lib import check
from .config import make_case

_pd = ctypes.POINTER(ctypes.c_double)


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_pd)


class ChannelCase:
    """One flat-channel case resident on the current CUDA device."""

    def __init__(self, **params):
        self.lib = _lib.load()
        self.params = dict(params)
        self.case = make_case(**params)
        h = ctypes.c_void_p()
        check(self.lib.tg_create(ctypes.byref(self.case), ctypes.byref(h)))
        self.h = h
        d = (ctypes.c_int * 6)()
        check(self.lib.tg_get_dims(self.h, d))
        self.nx, self.ny, self.nz, self.nxh, self.nyc, self.M = list(d)
        self.nphase = self.case.nphase

    # ---- lifetime
    def close(self):
        if getattr(self, "h", None):
            check(self.lib.tg_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(self.lib.tg_synchronize(self.h))

    def set_stream(self, stream_ptr: int):
        check(self.lib.tg_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    # ---- operators
    def operators(self) -> Tuple[np.ndarray, np.ndarray]:
        D1 = np.zeros((self.nz, self.nz))
        D2 = np.zeros((self.nz, self.nz))
        check(self.lib.tg_get_operators(self.h, _p(D1), _p(D2)))
        return D1, D2

    def decomposition(self, which: int) -> dict:
        n = self.nz
        out = {k: np.zeros((n, n)) for k in ("E", "Einv")}
        out.update({k: np.zeros(n) for k in ("lam", "fbb", "ftb", "fbf", "ftf")})
        check(self.lib.tg_get_decomposition(self.h, which, _p(out["E"]), _p(out["Einv"]), _p(out["lam"]),
                                            _p(out["fbb"]), _p(out["ftb"]), _p(out["fbf"]), _p(out["ftf"])))
        return out

    def set_decomposition(self, which: int, E, Einv, lam, fbb, ftb, fbf, ftf):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (E, Einv, lam, fbb, ftb, fbf, ftf)]
        check(self.lib.tg_set_decomposition(self.h, which, *[_p(a) for a in arrs]))

    # ---- state (Variable::Load / Save)
    def _shape(self, dim):
        return (dim, self.nxh, self.nyc, self.nz)

    def upload_state(self, uvw: np.ndarray, p: np.ndarray, phi: Optional[np.ndarray] = None, start_step: int = 0):
        u = np.ascontiguousarray(np.asarray(uvw, dtype=np.complex128).reshape(self._shape(3)))
        pp = np.ascontiguousarray(np.asarray(p, dtype=np.complex128).reshape(self._shape(1)))
        ph = None if phi is None else np.ascontiguousarray(np.asarray(phi, dtype=np.complex128).reshape(self._shape(1)))
        check(self.lib.tg_upload_state(self.h, _p(u.view(np.float64)), _p(pp.view(np.float64)),
                                       None if ph is None else _p(ph.view(np.float64)), int(start_step)))

    def download_state(self):
        u = np.zeros(self._shape(3), dtype=np.complex128)
        p = np.zeros(self._shape(1), dtype=np.complex128)
        ph = np.zeros(self._shape(1), dtype=np.complex128) if self.nphase > 1 else None
        check(self.lib.tg_download_state(self.h, _p(u.view(np.float64)), _p(p.view(np.float64)),
                                         None if ph is None else _p(ph.view(np.float64))))
        return u, p, ph

    # ---- time loop
    def set_time(self, step: int, time: float, dt: float, alternation: bool):
        check(self.lib.tg_set_time(self.h, int(step), float(time), float(dt), int(bool(alternation))))

    def get_time(self) -> dict:
        st, al, fw = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        t, dt, cfl = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(self.lib.tg_get_time(self.h, ctypes.byref(st), ctypes.byref(t), ctypes.byref(dt), ctypes.byref(al),
                                   ctypes.byref(fw), ctypes.byref(cfl)))
        return dict(step=st.value, time=t.value, dt=dt.value, alternation=bool(al.value), isforward=bool(fw.value),
                    cfl=cfl.value)

    def run_steps(self, nsteps: int, maxstep: int = 2 ** 30, maxcfl: float = 1e300,
                  features: Optional[np.ndarray] = None) -> int:
        done = ctypes.c_int()
        check(self.lib.tg_run_steps(self.h, int(nsteps), int(maxstep), float(maxcfl), _p(features),
                                    ctypes.byref(done)))
        return done.value

    def swirling_strength(self) -> np.ndarray:
        """FlatChannelPostprocessor: lambda_ci of the current state, (Nz, Ny, Nx) FP64."""
        out = np.zeros((self.nz, self.ny, self.nx))
        check(self.lib.tg_swirling_strength(self.h, _p(out)))
        return out

    def set_graphs(self, enable: bool):
        """Replay whole RK3 steps of run_steps as CUDA graphs (default) or not."""
        check(self.lib.tg_set_graphs(self.h, int(bool(enable))))

    def set_zsolver(self, solver: str):
        """Products of the dense Helmholtz solves in mixed precision: "dmma"
        (FP64 tensor cores) or "islice" (exact int8 slices on the tcgen05
        tensor cores)."""
        check(self.lib.tg_set_zsolver(self.h, {"dmma": 0, "islice": 1}[solver]))

    def autotune(self, cache_path: Optional[str] = None) -> dict:
        """Pick the z-operator GEMM row tiling for this grid and GPU (timed, or
        read from the JSON cache at cache_path) and apply it; returns the
        m-tiles per CTA and row tiles of the dense and the folded kernel."""
        t = (ctypes.c_int * 4)()
        path = None if cache_path is None else os.fsencode(cache_path)
        check(self.lib.tg_autotune(self.h, path, t))
        return dict(mt_dense=t[0], tiles_dense=t[1], mt_folded=t[2], tiles_folded=t[3])

    def features(self) -> np.ndarray:
        f = np.zeros(_lib.TG_NFEATURE)
        check(self.lib.tg_features(self.h, _p(f)))
        return f

    # ---- kernel-class timing
    def profile_begin(self):
        check(self.lib.tg_profile_begin(self.h))

    def profile_end(self) -> dict:
        n = _lib.TG_PROF_NCAT
        ms, by, fl = (np.zeros(n) for _ in range(3))
        cnt = np.zeros(n, dtype=np.int32)
        check(self.lib.tg_profile_end(self.h, n, _p(ms), _p(by), _p(fl), cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        xf = np.zeros(n)
        check(self.lib.tg_profile_executed(self.h, n, _p(xf)))
        return {name: dict(ms=float(ms[i]), bytes=float(by[i]), flops=float(fl[i]), xflops=float(xf[i]),
                           count=int(cnt[i]))
                for i, name in enumerate(_lib.PROF_NAMES)}

    # ---- plugin methods
    def carrier_predict(self, stage): check(self.lib.tg_carrier_predict(self.h, int(stage)))
    def carrier_correct(self, stage): check(self.lib.tg_carrier_correct(self.h, int(stage)))
    def scalar_predict(self, stage): check(self.lib.tg_scalar_predict(self.h, int(stage)))
    def scalar_correct(self, stage): check(self.lib.tg_scalar_correct(self.h, int(stage)))

    # ---- field-container primitives on device pointers
    def dft_forward(self, phys_ptr: int, spec_ptr: int, dim: int, fp32: bool = False):
        fn = self.lib.tg_dft_forward_f32 if fp32 else self.lib.tg_dft_forward_f64
        check(fn(self.h, ctypes.c_void_p(phys_ptr), ctypes.c_void_p(spec_ptr), int(dim)))

    def dft_backward(self, spec_ptr: int, phys_ptr: int, dim: int, fp32: bool = False):
        fn = self.lib.tg_dft_backward_f32 if fp32 else self.lib.tg_dft_backward_f64
        check(fn(self.h, ctypes.c_void_p(spec_ptr), ctypes.c_void_p(phys_ptr), int(dim)))

    def dft_forward_planes(self, phys_ptr: int, spec_ptr: int, planes: int, fp32: bool = False):
        """Forward x/y transforms of `planes` physical z planes (a z-slab)."""
        check(self.lib.tg_dft_forward_planes(self.h, ctypes.c_void_p(phys_ptr), ctypes.c_void_p(spec_ptr),
                                             int(planes), int(bool(fp32))))

    def dft_backward_planes(self, spec_ptr: int, phys_ptr: int, planes: int, fp32: bool = False):
        """Backward y/x transforms of `planes` spectral z planes (a z-slab)."""
        check(self.lib.tg_dft_backward_planes(self.h, ctypes.c_void_p(spec_ptr), ctypes.c_void_p(phys_ptr),
                                              int(planes), int(bool(fp32))))

    def multiply(self, A: np.ndarray, in_ptr: int, out_ptr: int, dim: int):
        A = np.ascontiguousarray(A, dtype=np.float64)
        check(self.lib.tg_multiply(self.h, _p(A), ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), int(dim)))

    def helmholtz(self, which: int, stage: int, rhs_ptr: int, out_ptr: int):
        check(self.lib.tg_helmholtz(self.h, int(which), int(stage), ctypes.c_void_p(rhs_ptr),
                                    ctypes.c_void_p(out_ptr)))


def operators_host(nz: int, mapping: int = 0, coef: float = 0.0):
    lib = _lib.load()
    D1 = np.zeros((nz, nz))
    D2 = np.zeros((nz, nz))
    check(lib.tg_operators_host(nz, mapping, coef, _p(D1), _p(D2)))
    return D1, D2


def decomposition_host(nz: int, bc, mapping: int = 0, coef: float = 0.0) -> dict:
    lib = _lib.load()
    bca = np.ascontiguousarray(bc[:4], dtype=np.float64)
    out = {k: np.zeros((nz, nz)) for k in ("E", "Einv")}
    out.update({k: np.zeros(nz) for k in ("lam", "fbb", "ftb", "fbf", "ftf")})
    check(lib.tg_decomposition_host(nz, mapping, coef, _p(bca), _p(out["E"]), _p(out["Einv"]), _p(out["lam"]),
                                    _p(out["fbb"]), _p(out["ftb"]), _p(out["fbf"]), _p(out["ftf"])))
    return out


def to_slab(ref: np.ndarray) -> np.ndarray:
    """(dim, Nxh, Nyc, Nz) reference layout -> (dim, Nz, M) z-slab layout."""
    d, nxh, nyc, nz = ref.shape
    return np.ascontiguousarray(ref.reshape(d, nxh * nyc, nz).transpose(0, 2, 1))


def from_slab(slab: np.ndarray, nxh: int, nyc: int) -> np.ndarray:
    d, nz, M = slab.shape
    return np.ascontiguousarray(slab.transpose(0, 2, 1).reshape(d, nxh, nyc, nz))


def run_ensemble(cases, nsteps: int, maxstep: int = 2 ** 30, maxcfl: float = 1e300):
    """tg_run_ensemble: nsteps RK3 steps of independent cases stepped together
    (each on its own stream); returns the steps each case took."""
    lib = _lib.load()
    n = len(cases)
    handles = (ctypes.c_void_p * n)(*[c.h.value if isinstance(c.h, ctypes.c_void_p) else c.h for c in cases])
    done = (ctypes.c_int * n)()
    check(lib.tg_run_ensemble(handles, n, int(nsteps), int(maxstep), float(maxcfl), done))
    return list(done)
