#!/usr/bin/env python3
"""RK3 steps/s of TURBID's flat-channel substep on B200.

Workload (default "cfg3"): 256x256x257 Fourier-Chebyshev grid, oscillatory
boundary layer Re_delta = 800 with one fine-sediment scalar (Ws = 5e-4,
Sc = 0.5, Boussinesq coupling s = 2.65, C = 1e-3, erosion/deposition bottom),
dt = 2 pi/2000, mixed precision (FP32 transforms and nonlinear products, FP64
z-operators and Helmholtz solves).  Synthetic seeded initial state (the
reference has no public dataset).  One "step" = one full RK3 step (3 stages
of both phases).  All fields (>= 300 MB of spectral state plus physical
buffers) exceed the 126 MB L2, so no explicit L2 flush is done between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Rank 0 prints one JSON line.  With N > 1 (torchrun) every rank runs an
independent replica of the case (the path has no cross-case exchange), and
value = total steps of all ranks / max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK3 steps/sec @256x256x257, mixed vs FP64 GPU at rel-L2<=1e-5; HBM GB/s"

WORKLOADS = {
    # name: grid, physics, precision
    "cfg3": dict(nx=256, ny=256, nz=257, nphase=2, reynolds=800.0, precision="mixed"),
    "cfg2": dict(nx=128, ny=128, nz=129, nphase=2, reynolds=800.0, precision="fp64"),
    "cfg1": dict(nx=32, ny=32, nz=65, nphase=1, reynolds=180.0, precision="fp64"),
    "cfg5": dict(nx=512, ny=256, nz=257, nphase=2, reynolds=1000.0, precision="mixed", lx=8 * math.pi),
    "small": dict(nx=64, ny=64, nz=65, nphase=2, reynolds=800.0, precision="mixed"),
    # batched ensemble: 16 cases, grids drawn between 64^2x65 and 192^2x193 (see ensemble_params)
    "cfg4": dict(nx=64, ny=64, nz=65, nphase=2, reynolds=800.0, precision="mixed"),
}


def replica_max(v: float, dist=None, device: str = "cpu") -> float:
    """The maximum of a per-rank value over all ranks (the slowest replica's
    time); dist is torch.distributed (NCCL on the GPU box, gloo in tests)."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(steps_per_rank: int, ms_max: float, world: int) -> float:
    """Whole-job throughput of N independent replicas: all ranks' steps over
    the slowest rank's device time."""
    return steps_per_rank * world / (ms_max * 1e-3)


def ensemble_params(count: int = 16, seed: int = 4, smooth_only: bool = True) -> list:
    """Uneven grids and parameters drawn from a seed: Nx = Ny even in [64, 192]
    with prime factors up to 7 (the FFT-friendly lengths a spectral case uses;
    smooth_only=False draws any even length: the library runs those too, a
    prime factor above 13 through a direct-DFT pass, several times slower),
    Nz = Nx + 1, Re ~ U[400, 1000], Ws ~ logU[1e-4, 1e-3], Schmidt 0.5."""
    def smooth(n):
        for q in (2, 3, 5, 7):
            while n % q == 0:
                n //= q
        return n == 1
    sizes = [n for n in range(64, 193, 2) if smooth(n) or not smooth_only]
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(sizes[rng.integers(0, len(sizes))])
        p = case_params("cfg4")
        p.update(nx=n, ny=n, nz=n + 1, reynolds=float(rng.uniform(400.0, 1000.0)),
                 settling=float(10 ** rng.uniform(-4.0, -3.0)))
        out.append(p)
    return out


def ensemble_arm(args):
    """16 independent cases stepped together (tg_run_ensemble, one stream and
    one step graph per case) against the same cases stepped one after another."""
    import torch
    import turbid_b200 as tb
    from turbid_b200 import synthetic, _lib
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    plist = ensemble_params()
    lib = _lib.load()
    cases, streams = [], []
    for i, p in enumerate(plist):
        s = torch.cuda.Stream()
        c = tb.ChannelCase(**dict(p, precision=args.precision or p["precision"]))
        c.set_stream(s.cuda_stream)
        uvw, pr, phi = synthetic.initial_state(seed=100 + i, **p)
        c.upload_state(uvw, pr, phi)
        c.run_steps(args.warmup)
        cases.append(c)
        streams.append(s)
    torch.cuda.synchronize()
    base = torch.cuda.Stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(base)
        for s in streams:
            s.wait_event(e0)
        fn()
        for s in streams:
            ev = torch.cuda.Event()
            ev.record(s)
            base.wait_event(ev)
        e1.record(base)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    sampler = ClockSampler(0)
    sampler.start()
    l0 = lib.tg_launch_count()
    ms = timed(lambda: tb.run_ensemble(cases, args.steps))
    launches = lib.tg_launch_count() - l0
    clocks = sampler.stop()
    ms_seq = timed(lambda: [c.run_steps(args.steps) for c in cases])
    steps = args.steps * len(cases)
    points = sum(p["nx"] * p["ny"] * p["nz"] for p in plist)
    line = {"metric": "ensemble case-steps/sec (16 cases, 64^2x65 .. 192^2x193, sediment)",
            "value": steps / (ms * 1e-3), "unit": "case-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 transforms/products + f64 z-solves", "data": "synthetic",
            "config": {"workload": "cfg4 batched ensemble", "cases": [(p["nx"], p["nz"]) for p in plist],
                       "grid_points": points, "precision": args.precision or "mixed",
                       "parallelism": "single GPU, one stream and one step graph per case"},
            "sequential_case_steps_per_s": steps / (ms_seq * 1e-3),
            "gpu_launches": launches, "clocks": clocks}
    print(json.dumps(line), flush=True)
    for c in cases:
        c.close()


def case_params(name: str) -> dict:
    w = dict(WORKLOADS[name])
    p = dict(lx=4 * math.pi, ly=2 * math.pi, dt=2 * math.pi / 2000, froude=1.0, averaged_concentration=1e-3,
             specific_gravity=2.65, affected_by_scalar=1, bc_u=[1, 0, 0, 1, 0], bc_v=[1, 0, 0, 1, 0],
             bc_w=[1, 0, 1, 0, 0], bc_p=[0, 1, 0, 1, 0], force_type=2, force_direction=[0, 1],
             force_amplitude=[0, 1], schmidt=0.5, settling=5e-4, erosion_rate=1e-4, critical_shear=2e-4,
             scalar_bc=1)
    if w["nphase"] == 1:
        p["bc_u"] = p["bc_v"] = [1, 0, 0, 1, 0]
    p.update(w)
    return p


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for i, n in enumerate(names):
                if r[5 + i].strip().lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def fp64_gemm_peak(torch) -> float:
    """cuBLAS DGEMM TFLOP/s measured in this run (the FP64 tensor-core reference)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def traffic_summary() -> dict:
    """Per-launch DRAM bytes of each kernel class from the committed ncu
    captures (profiles/traffic.json; its "note" says which launch each is)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return {k: v for k, v in json.load(f).items() if k != "note"}
    except Exception:
        return {}


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 oracle port of the reference path on the host cores
# ---------------------------------------------------------------------------
def cpu_step_rate(wname: str, nsteps_max: int, budget_s: float, warmup: int):
    from oracle import turbid_oracle as O
    from turbid_b200 import synthetic
    p = case_params(wname)
    keys = [f for f in O.CaseConfig.__dataclass_fields__ if f in p]
    cfg = O.CaseConfig(**{k: p[k] for k in keys})
    uvw, pr, phi = synthetic.initial_state(seed=1234, **p)
    t0 = time.perf_counter()
    sol = O.OracleSolver(cfg, uvw, pr, phi if cfg.nphase > 1 else None)
    setup = time.perf_counter() - t0
    for _ in range(min(warmup, 1)):
        sol.run_step()
    done, t0 = 0, time.perf_counter()
    while done < nsteps_max:
        sol.run_step()
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return done / el, done, el, setup


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = int(os.environ.get("TURBID_ORACLE_THREADS", os.cpu_count() or 1))
    rate, done, el, setup = cpu_step_rate(args.workload, args.steps, args.cpu_budget, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": done, "steps_requested": args.steps, "warmup": min(args.warmup, 1), "ms_per_step": 1e3 / rate,
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.workload} " + wdesc(args.workload), "precision": "fp64 (CPU)"},
        "cpu_baseline": {"value": rate, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": f"{done} RK3 step(s) of the full grid after min(W,1) warm-up step(s), "
                                   f"{el:.1f} s timed (budget {args.cpu_budget:.0f} s); numpy/scipy FP64 "
                                   f"restatement of the reference path (the reference needs MPI/Fortran/MKL "
                                   f"and does not build here)"},
        "e2e": {"value": rate, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def wdesc(name):
    p = WORKLOADS[name]
    return f"{p['nx']}x{p['ny']}x{p['nz']} Re{int(p['reynolds'])} {'+sediment' if p['nphase'] > 1 else ''}"


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def our_arm(args):
    import torch
    import turbid_b200 as tb
    from turbid_b200 import synthetic, _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    params = case_params(args.workload)
    prec = args.precision or params["precision"]
    uvw0, p0, phi0 = synthetic.initial_state(seed=1234, **params)
    lib = _lib.load()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        return replica_max(v, dist, "cuda")

    # a dedicated stream: whole steps are then replayed as CUDA graphs (the
    # legacy default stream cannot be captured); events are recorded on it
    stream = torch.cuda.Stream()
    case = tb.ChannelCase(**dict(params, precision=prec))
    case.set_stream(stream.cuda_stream)
    if args.zsolver and prec == "mixed":
        case.set_zsolver(args.zsolver)
    case.upload_state(uvw0, p0, phi0)
    # z-operator GEMM row tiling picked by the library's own autotuner (timed
    # here, before the warm-up; the fields do not depend on it)
    tiling = case.autotune(None)
    case.run_steps(args.warmup)
    barrier()

    # ---- device-timed steps (state resident in HBM)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    l0 = lib.tg_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    done = case.run_steps(args.steps)
    e1.record(stream)
    barrier()
    launches = lib.tg_launch_count() - l0
    clocks = sampler.stop() if sampler else None
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = replica_rate(done, ms, world)

    # ---- kernel classes of the same workload (separate pass, CUDA events per launch)
    case.profile_begin()
    case.run_steps(args.prof_steps)
    prof = case.profile_end()
    peaks = measured_peaks()

    # ---- e2e through the C ABI with host buffers: H2D of the restart state,
    # K steps each returning the 50-double feature vector, D2H of the state
    pin = {k: torch.from_numpy(v.view(np.float64)).pin_memory() for k, v in
           (("u", np.ascontiguousarray(uvw0)), ("p", np.ascontiguousarray(p0)), ("c", np.ascontiguousarray(phi0)))}
    outs = {k: torch.empty_like(v).pin_memory() for k, v in pin.items()}
    feats = np.zeros(50)

    def ptr(t):
        import ctypes
        return ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))

    barrier()
    t0 = time.perf_counter()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    tb._lib.check(lib.tg_upload_state(case.h, ptr(pin["u"]), ptr(pin["p"]), ptr(pin["c"]), 0))
    n_e2e = 0
    for _ in range(args.steps):
        n_e2e += case.run_steps(1, features=feats)
    tb._lib.check(lib.tg_download_state(case.h, ptr(outs["u"]), ptr(outs["p"]), ptr(outs["c"])))
    f1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(max(f0.elapsed_time(f1), (time.perf_counter() - t0) * 1e3))
    state_bytes = sum(v.numel() * 8 for v in pin.values())
    e2e = {"value": n_e2e * world / (e2e_ms * 1e-3), "unit": "steps/s",
           "h2d_bytes_per_step": state_bytes / max(n_e2e, 1) + 16,
           "d2h_bytes_per_step": state_bytes / max(n_e2e, 1) + 400,
           "what": "tg_upload_state from pinned host (restart layout) + K x tg_run_steps(1) with the 400-byte "
                   "feature vector read back each step + tg_download_state, all inside the timed region"}

    # ---- accuracy vs the FP64 GPU path + FP64 GPU rate (same seed, same steps)
    acc = None
    fp64_rate = None
    if prec == "mixed" and not args.skip_accuracy and args.acc_steps > 0:
        ref = tb.ChannelCase(**dict(params, precision="fp64"))
        ref.set_stream(stream.cuda_stream)
        ref.upload_state(uvw0, p0, phi0)
        ref.run_steps(args.warmup)
        barrier()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        nd = ref.run_steps(args.steps)
        g1.record(stream)
        barrier()
        fp64_rate = nd / (g0.elapsed_time(g1) * 1e-3)
        # same initial state, same number of steps in both precisions
        nacc = args.acc_steps
        for c in (case, ref):
            c.upload_state(uvw0, p0, phi0)
            c.run_steps(nacc)
        a_u, a_p, a_c = case.download_state()
        b_u, b_p, b_c = ref.download_state()

        def rl(a, b):
            return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
        acc = {"steps": nacc, "u": rl(a_u[0], b_u[0]), "v": rl(a_u[1], b_u[1]), "w": rl(a_u[2], b_u[2]),
               "p": rl(a_p, b_p)}
        if params["nphase"] > 1:
            acc["c"] = rl(a_c, b_c)
        acc["max"] = max(v for k, v in acc.items() if k != "steps")
        acc["tolerance"] = 1e-5
        ref.close()

    # ---- roofline of the dominant kernel class
    steps_p = max(args.prof_steps, 1)
    if not any(v["ms"] > 0 for v in prof.values()):
        prof = {"zgemm": {"ms": 0.0, "bytes": 0.0, "flops": 0.0, "count": 0}}
    dom = max(prof, key=lambda k: prof[k]["ms"])
    d = prof[dom]
    traffic = traffic_summary().get(args.workload, {}).get(prec, {}).get(dom)
    if d["ms"] <= 0:
        roof = None
    elif dom == "zgemm":
        peak = fp64_gemm_peak(torch)
        achieved = d["flops"] / (d["ms"] * 1e-3) / 1e12
        executed = d.get("xflops", d["flops"]) / (d["ms"] * 1e-3) / 1e12
        roof = {"kernel": "zgemm_dense_kernel / zgemm_sym_kernel (FP64 DMMA z-operator GEMMs; the mixed mode's "
                          "dense solves run on the int8-slice kernels, class 'islice' of kernels)",
                "bound": "tensor",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "flops": "algorithmic: 4 Nz^2 M per component application (the dense FP64 product the reference "
                         "performs); the folded and split kernels execute about half of that",
                "executed_tflops": executed, "executed_frac": executed / peak,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                "per_launch_flops": d["flops"] / max(d["count"], 1), "traffic": traffic}
    else:
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = d["bytes"] / (d["ms"] * 1e-3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback",
                "traffic": traffic}
    hbm = peaks.get("hbm_gbs", 6650.0)
    kernels = {}
    for k, v in prof.items():
        if v["count"] == 0:
            continue
        gbs = v["bytes"] / (v["ms"] * 1e-3) / 1e9 if v["ms"] > 0 else 0.0
        ent = {"ms_per_step": v["ms"] / steps_p, "launches_per_step": v["count"] / steps_p, "GB/s": gbs,
               "hbm_frac": gbs / hbm}
        tr = traffic_summary().get(args.workload, {}).get(prec, {}).get(k)
        if tr:
            ent["traffic_per_launch"] = tr
        if v["flops"] and k == "islice":
            # FP64-equivalent: the dense products these int8 slices stand for
            ent["fp64_equivalent_TFLOP/s"] = v["flops"] / (v["ms"] * 1e-3) / 1e12
        elif v["flops"]:
            ent["TFLOP/s"] = v["flops"] / (v["ms"] * 1e-3) / 1e12
            ent["executed_TFLOP/s"] = v.get("xflops", v["flops"]) / (v["ms"] * 1e-3) / 1e12
        kernels[k] = ent

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            rate, n, el, setup = cpu_step_rate(args.workload, 1, args.cpu_budget, 0)
            cpu = {"value": rate, "unit": "steps/s",
                   "cores": int(os.environ.get("TURBID_ORACLE_THREADS", os.cpu_count() or 1)), "kind": "port",
                   "sample": f"{n} full RK3 step(s) of the same grid ({el:.1f} s), numpy/scipy FP64 restatement "
                             f"of the reference path on all host threads"}
        except Exception as exc:  # the baseline is a report, never a reason to lose the GPU line
            cpu = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"failed: {exc}"}
    case.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / max(done, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 transforms/products + f64 z-solves" if prec == "mixed" else "f64",
            "data": "synthetic (seeded Stokes profile + divergence-free perturbation, 10% scalar noise)",
            "config": {"workload": f"{args.workload} {wdesc(args.workload)}", "precision": prec,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (no flush)",
                       "zsolver": (args.zsolver or "library default") if prec == "mixed" else "dmma",
                       "gemm_tiling": "autotuned: dense {mt_dense} m-tiles x {tiles_dense} row tiles, "
                                      "folded {mt_folded} x {tiles_folded}".format(**tiling)},
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks, "roofline": roof,
            "cpu_baseline": cpu, "accuracy_vs_fp64_gpu": acc, "fp64_gpu_steps_per_s": fp64_rate,
            "kernels": kernels,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg3", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default=None, choices=[None, "fp64", "mixed"])
    ap.add_argument("--zsolver", default=None, choices=[None, "dmma", "islice"],
                    help="products of the dense Helmholtz solves in mixed precision (default: the library's)")
    ap.add_argument("--prof-steps", type=int, default=3)
    ap.add_argument("--acc-steps", type=int, default=None,
                    help="steps of the mixed vs FP64 comparison (default 100; 5 for cfg5)")
    ap.add_argument("--skip-accuracy", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=60.0)
    args = ap.parse_args()
    if args.acc_steps is None:
        args.acc_steps = 5 if args.workload == "cfg5" else 100
    if args.impl == "reference":
        reference_arm(args)
    elif args.workload == "cfg4":
        ensemble_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()
