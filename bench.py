#!/usr/bin/env python
"""Throughput of the projection-method time step on B200 (Mcell-steps/s).

Workload: the 128^3 lid-driven cavity (Re=1000, dt=5e-4, zero initial
fields), one step = one pass of the loop body (predictor, red-black SOR
pressure solve to zeta = 1e-4, projection + direct forcing + force integral,
boundary conditions).  The timed region runs exactly --steps steps starting
from the initial state (after --warmup untimed steps and a reset); by
default 500 steps, i.e. the whole case.  The mixed-precision step is the
headline; the plain FP64 step runs on the same steps for the speed-up and
the relative L2 error.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--gpus N > 1 runs one independent replica per GPU (the case does not shard
across GPUs); value = total cells * steps / max-over-ranks device time.
--impl reference times the CPU restatement of the reference's own algorithm
(lexicographic SOR with the reference's OpenMP loop schedule) on the host
cores, rank 0 only.

The "adjoint" object (rank 0, one GPU) gives the second half of the metric:
wall time of ntcfd_adjoint over K = 200 steps of the cylinder case (32x96x96,
checkpoints every 20 steps) divided by the device time of the plain K-step
forward, and the agreement of its gradients (inflow speed, inflow angle, a
random direction of the body force) with central differences.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s mixed-prec vs FP64 plain at ≤1e-6 rel L2; adjoint/forward cost"
UNIT = "Mcell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=None, help="cavity cells per side (default: the case's)")
    ap.add_argument("--case", choices=("c2", "c1"), default="c2",
                    help="c2: 128^3 cavity, Re=1000, dt=5e-4 (the headline); c1: 40^3, Re=100, dt=1e-3")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--cycle", type=int, default=8,
                    help="mixed path: FP32 sweeps per FP64 defect-correction cycle")
    ap.add_argument("--eager", action="store_true",
                    help="launch kernels one by one instead of CUDA graphs (for ncu)")
    ap.add_argument("--sor-path", choices=("auto", "streaming", "resident"), default="auto")
    ap.add_argument("--no-roofline", action="store_true", help="skip the standalone kernel timing")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint cost/accuracy leg")
    ap.add_argument("--no-fd", action="store_true", help="skip the finite-difference check of the adjoint")
    a = ap.parse_args()
    # the cavity of the case: Reynolds number, time step (a Fortran default-real literal) and size
    a.Re, a.dt = (1000.0, 5e-4) if a.case == "c2" else (100.0, 1e-3)
    if a.n is None:
        a.n = 128 if a.case == "c2" else 40
    return a


# ------------------------------------------------------------------ ranks
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def aggregate(values, op):
    """Reduces one float per rank (max or sum) over torch.distributed when
    it is initialised; identity on a single process."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(values)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(values)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                mx = float(f[2].split()[0])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ our arm
def cavity_case(n, precision, device, args):
    from ntustcfdlab_b200 import cases
    c = cases.cavity(n, args.Re, args.dt, 500, precision=precision)
    c.params.device = device
    c.params.mixed_cycle = args.cycle if precision == 1 else 0
    c.params.eager = 1 if args.eager else 0
    c.params.sor_path = {"auto": 0, "streaming": 1, "resident": 2}[args.sor_path]
    return c


def reset(s):
    z = np.zeros(s.halo_shape, order="F")
    s.set_state(z, z, z, z)
    s.boundary_conditions()


def timed_run(case, K, W, sampler_index=None):
    """W warm-up steps, reset to the initial state, then K device-timed steps."""
    from ntustcfdlab_b200.solver import Solver
    import torch
    s = Solver(case.params, case.grid)
    s.boundary_conditions()
    if W > 0:
        s.step(W)
    reset(s)
    torch.cuda.synchronize()
    barrier()
    clocks = None
    if sampler_index is not None:
        with ClockSampler(sampler_index) as cs:
            info, rc = s.step(K)
        clocks = cs.summary()
    else:
        info, rc = s.step(K)
    torch.cuda.synchronize()
    barrier()
    ms = s.last_step_ms()
    return s, info, rc, ms, clocks


def e2e_run(case, K, isto=100):
    """The same K steps through the C-ABI with host buffers: upload the
    initial state from pinned host memory, one ntcfd_step(ctx, 1, &info) per
    step (info back to the host every step, as the reference driver prints
    it), centred output fields to the host every `isto` steps
    (filereachtime cadence, main.f90:317-324) through ntcfd_output_async, so
    the copy overlaps the following steps, and the final state."""
    import torch
    from ntustcfdlab_b200.solver import Solver
    s = Solver(case.params, case.grid)
    s.boundary_conditions()
    s.step(2)                       # graph instantiation outside the timed region
    shape = s.halo_shape
    n_halo = int(np.prod(shape))
    n_in = int(np.prod(s.inner_shape))
    pin = lambda n: torch.zeros(n, dtype=torch.float64, pin_memory=True).numpy()
    state = [pin(n_halo).reshape(shape, order="F") for _ in range(4)]
    outs = [pin(n_in).reshape(s.inner_shape, order="F") for _ in range(4)]
    back = [pin(n_halo).reshape(shape, order="F") for _ in range(4)]
    from ntustcfdlab_b200.abi import dptr
    lib, h = s.lib, s.h
    from ntustcfdlab_b200.abi import NtcfdStepInfo
    info = NtcfdStepInfo()
    lib.ntcfd_output_async(h, *[dptr(a) for a in outs])   # allocates the output buffers
    lib.ntcfd_output_wait(h)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lib.ntcfd_set_state(h, *[dptr(a) for a in state])
    lib.ntcfd_apply_bc(h)
    h2d = 4 * n_halo * 8
    d2h = 0
    pending = False
    for k in range(1, K + 1):
        rc = lib.ntcfd_step(h, 1, info)
        if rc < 0:
            raise RuntimeError(s._err())
        d2h += 40  # the step record (StepRec) crosses back every step
        if k % isto == 0:           # waits for the previous output first
            if lib.ntcfd_output_async(h, *[dptr(a) for a in outs]) != 0:
                raise RuntimeError(s._err())
            pending = True
            d2h += 4 * n_in * 8
    if pending and lib.ntcfd_output_wait(h) != 0:
        raise RuntimeError(s._err())
    lib.ntcfd_get_state(h, *[dptr(a) for a in back])
    d2h += 4 * n_halo * 8
    t1 = time.perf_counter()
    s.close()
    return (t1 - t0), h2d, d2h


def cpu_baseline_from(s_gpu, case, seconds, threads=None):
    """Oracle (the CPU restatement of the reference's algorithm, lexicographic
    SOR with the reference's OpenMP schedule, all host threads unless
    `threads` is given) on a bounded sample: consecutive steps from the device
    state at the end of the timed run, until `seconds` of CPU time have
    passed."""
    from oracle import cpu_oracle
    from ntustcfdlab_b200.abi import SOR_LEX, params_copy
    threads = threads or os.cpu_count() or 1
    o = cpu_oracle.Oracle(params_copy(case.params, sor_order=SOR_LEX), case.grid, threads=threads)
    o.initial_conditions()
    for k, a in zip("uvwp", s_gpu.get_state()):
        o.set(k, a)
    o.boundary_conditions()
    t0 = time.perf_counter()
    steps = sweeps = 0
    while True:
        inf = o.step(1)[0]
        steps += 1
        sweeps += inf.sor_iters
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 50:
            break
    return case.cells * steps / el / 1e6, threads, steps, sweeps, el


def roofline(s, case, path, reps=20):
    """Dominant kernel: the SOR sweeps.  Algorithmic bytes: 3 S per cell per
    full red+black sweep (read e, d and rd, write e of every cell once; S = 4 B
    mixed, 8 B FP64).  Streaming path: one launch = one colour = 1.5 S per
    cell.  Resident path: one launch runs `resident_sweeps` sweeps (timed
    standalone, zeta = 0).

    `traffic` is the DRAM traffic of one launch of the same kernel on the same
    grid from an ncu capture (profiles/sor_traffic.json).  `bound` follows
    from it: a kernel whose DRAM traffic is well below its algorithmic bytes
    works out of shared memory and L2, so the HBM roofline does not bind it
    ("on-chip"; the resident kernel is then bound by its grid barriers and
    instruction issue); otherwise "hbm".  Both fractions are reported: the
    algorithmic one (`frac`) and the DRAM one (`dram_frac`).

    `per_kernel` gives each stencil kernel's algorithmic bytes per launch
    over its CUDA-event time as a fraction of the measured HBM bandwidth."""
    kt = s.time_kernels(reps)
    S = 4 if case.params.precision == 1 else 8
    N = case.cells
    if path == 2 and kt["resident_ms"] > 0:
        kernel = "k_sor_resident (all sweeps of a correction cycle, e in shared memory)"
        alg = 3 * S * N * kt["resident_sweeps"]
        ms = kt["resident_ms"]
    else:
        kernel = "k_sweep (one colour of a red-black SOR sweep)"
        alg = 1.5 * S * N
        ms = kt["sweep_ms"]
    ach = alg / (ms * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    traffic = None
    tp = os.path.join(ROOT, "profiles", "sor_traffic.json")
    if os.path.exists(tp):
        try:
            tr = json.load(open(tp))
            key = f"{case.params.nx}:{S}:{path}"
            if key in tr:
                traffic = tr[key]["dram_bytes_per_launch"]
        except Exception:
            traffic = None
    dram_ach = traffic / (ms * 1e-3) / 1e9 if traffic else None
    bound = "hbm" if traffic is None or traffic >= 0.5 * alg else "on-chip"
    # algorithmic bytes per cell of the other stencil kernels (FP64 state arrays)
    les = 8 if case.params.LES else 0
    per_cell = {"predictor_ms": 48 + les, "rhs_ms": 32, "defect_ms": 16 + 2 * S, "project_ms": 64,
                "sweep_ms": 1.5 * S}
    per_kernel = {}
    for k, b in per_cell.items():
        t = kt.get(k, 0.0)
        if t > 0:
            per_kernel[k[:-3]] = {"ms": round(t, 5), "bytes": b * N,
                                  "frac": round(b * N / (t * 1e-3) / 1e9 / peak, 3)}
    return {"kernel": kernel, "bound": bound, "achieved": round(ach, 1), "peak": peak,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "unit": "GB/s", "frac": round(ach / peak, 3), "traffic": traffic,
            "dram_achieved": round(dram_ach, 1) if dram_ach else None,
            "dram_frac": round(dram_ach / peak, 4) if dram_ach else None,
            "algorithmic_bytes_per_launch": alg, "avg_launch_ms": ms,
            "per_kernel": per_kernel,
            "kernel_ms": {k: round(v, 5) for k, v in kt.items()}}


def adjoint_leg(device, fd=True, K=200, M=20):
    """Adjoint cost and accuracy on the cylinder case: J = mean cDrag over
    K steps from an impulsive start with the seeded body force, checkpoints
    every M steps.  Cost = wall time of ntcfd_adjoint / device time of the
    plain K-step forward (reference zeta 1e-4).  Accuracy = the adjoint
    (default adjoint stop rule) against central differences h = 1e-6 of
    K-step runs whose pressure solves run to zeta = 1e-12."""
    import math
    from ntustcfdlab_b200 import abi, cases
    from ntustcfdlab_b200.solver import Solver

    def case(prec, zeta=abi.f4(1e-4), U=1.0, theta_deg=0.0):
        kw = dict(zeta=zeta, itmax=200000 if zeta < 1e-6 else 3000, device=device)
        if prec == abi.MIXED:
            kw["mixed_cycle"] = 8
        return cases.c4(precision=prec, U=U, theta_deg=theta_deg, **kw)

    base = case(abi.FP64)
    nx, ny, nz = base.params.nx, base.params.ny, base.params.nz
    force = cases.body_force_c4((nx, ny, nz))
    s0 = Solver(base.params, base.grid)
    s0.set_state(*cases.uniform_inflow_state(base))
    s0.boundary_conditions()
    st = s0.get_state()
    s0.close()

    def solver(c, f=force):
        s = Solver(c.params, c.grid)
        s.build_mask_cylinder(c.mask["zc"], c.mask["yc"], c.mask["r"])
        s.set_state(*st)
        s.set_body_force(*f)
        return s

    out = {"case": "cylinder D=1, 32x96x96 (span x, y, z) uniform over 4x12x12, Re=100, dt=5e-3, "
                   "impulsive start, inflow w=1 on the Back wall, body force N(0,1e-3) seed "
                   f"{cases.C4_SEED}", "K": K, "M": M, "objective": "mean cDrag over the K steps",
           "adj_zeta": 1e-7, "adj_omega": 1.9}
    for prec, name in ((abi.MIXED, "mixed"), (abi.FP64, "fp64")):
        c = case(prec)
        s = solver(c)
        s.step(2)                          # graph instantiation
        s.set_state(*st)
        s.adjoint(K, M, w_drag=1.0, inflow=("Back", 2, 1))   # warm-up: workspace, kernel loading
        s.set_state(*st)
        info, rc = s.step(K)
        fwd = s.last_step_ms()
        s.set_state(*st)
        r = s.adjoint(K, M, w_drag=1.0, inflow=("Back", 2, 1))
        s.close()
        out[name] = {"forward_ms": round(fwd, 3), "adjoint_total_ms": round(r["total_ms"], 3),
                     "adjoint_over_forward": round(r["total_ms"] / fwd, 3),
                     "phases_ms": {"forward_pass": round(r["forward_ms"], 3),
                                   "recompute": round(r["recompute_ms"], 3),
                                   "adjoint_solves": round(r["solve_ms"], 3)},
                     "adjoint_sweeps": r["adj_sweeps"], "forward_sweeps": int(sum(i.sor_iters for i in info)),
                     "dJ_dU": r["dJ_dU"], "dJ_dtheta": r["dJ_dtheta"]}
    if fd:
        h = 1e-6
        tight = case(abi.FP64, zeta=1e-12)
        s = solver(tight)
        r = s.adjoint(K, M, w_drag=1.0, inflow=("Back", 2, 1))
        s.close()

        def J(U=1.0, th=0.0, f=force):
            s = solver(case(abi.FP64, zeta=1e-12, U=U, theta_deg=math.degrees(th)), f)
            info, rc = s.step(K)
            s.close()
            return sum(i.cDrag for i in info) / K

        gU = (J(U=1 + h) - J(U=1 - h)) / (2 * h)
        gth = (J(th=h) - J(th=-h)) / (2 * h)
        rng = np.random.default_rng(11)
        d = [rng.standard_normal(f.shape) for f in force]
        gf = (J(f=[a + h * e for a, e in zip(force, d)]) - J(f=[a - h * e for a, e in zip(force, d)])) / (2 * h)
        ga = sum(float(np.sum(a * e)) for a, e in zip(r["dJ_df"], d))
        out["fd_check"] = {"forward_zeta": 1e-12, "h": h,
                           "dJ_dU": [r["dJ_dU"], gU], "dJ_dtheta": [r["dJ_dtheta"], gth],
                           "dJ_df_dir": [ga, gf],
                           "rel_err": {"U": abs(r["dJ_dU"] - gU) / abs(gU),
                                       "theta": abs(r["dJ_dtheta"] - gth) / abs(gth),
                                       "force_dir": abs(ga - gf) / abs(gf)}}
    return out


def rel_l2(a, b):
    a = a[2:-2, 2:-2, 2:-2]
    b = b[2:-2, 2:-2, 2:-2]
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a - b))


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from ntustcfdlab_b200.abi import FP64, MIXED
    K, W = args.steps, max(args.warmup, 0)
    mixed = cavity_case(args.n, MIXED, local, args)
    s, info, rc, ms, clocks = timed_run(mixed, K, W, sampler_index=local)
    ms_max = aggregate(ms, "max")
    cells_total = mixed.cells * world
    value = cells_total * K / (ms_max * 1e-3) / 1e6
    sweeps = [i.sor_iters for i in info]
    launches = int(sum(i.launches for i in info))
    extra = {}
    if not args.no_fp64:
        f64 = cavity_case(args.n, FP64, local, args)
        s64, info64, _, ms64, _ = timed_run(f64, K, W)
        ms64_max = aggregate(ms64, "max")
        v64 = cells_total * K / (ms64_max * 1e-3) / 1e6
        st32, st64 = s.get_state(), s64.get_state()
        extra["fp64"] = {"value": round(v64, 2), "ms_per_step": ms64_max / K,
                         "sweeps_total": int(sum(i.sor_iters for i in info64))}
        extra["mixed_over_fp64"] = round(value / v64, 3)
        extra["rel_l2_mixed_vs_fp64"] = {k: rel_l2(a, b) for k, a, b in zip("uvwp", st32, st64)}
        s64.close()
    e2e = None
    if not args.no_e2e:
        t, h2d, d2h = e2e_run(mixed, K)
        t_max = aggregate(t, "max")
        e2e = {"value": round(cells_total * K / t_max / 1e6, 2), "unit": UNIT,
               "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
               "timing": "host wall clock around the synchronous C-ABI calls"}
    path = info[0].sor_path if info else 1
    rl = roofline(s, mixed, path) if rank == 0 and not args.no_roofline else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, thr, nst, nsw, el = cpu_baseline_from(s, mixed, args.cpu_seconds)
        cpu = {"value": round(v, 4), "unit": UNIT, "cores": thr, "kind": "port",
               "sample": (f"{nst} consecutive steps ({nsw} SOR sweeps, {el:.1f} s) of the same "
                          f"{args.n}^3 case from the device state after step {K}; lexicographic "
                          f"SOR with the reference's OpenMP schedule, {thr} threads")}
        # the same sample on one host thread (the reference's serial build)
        v1, _, nst1, nsw1, el1 = cpu_baseline_from(s, mixed, args.cpu_seconds / 2, threads=1)
        cpu["single_thread"] = {"value": round(v1, 4), "unit": UNIT, "cores": 1,
                                "sample": f"{nst1} consecutive steps ({nsw1} SOR sweeps, {el1:.1f} s)"}
    adj = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adj = adjoint_leg(local, fd=not args.no_fd)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (lid-driven cavity from rest, no dataset)",
            "config": {"workload": f"lid-driven cavity {args.n}^3, Re={args.Re:g}, dt={args.dt:g}, zeta=1e-4, "
                                   f"mixed precision (FP32 red-black SOR + FP64 defect correction "
                                   f"every {args.cycle} sweeps)",
                       "sor_path": {1: "streaming", 2: "resident"}.get(path, str(path)),
                       "launch": "eager" if args.eager else "cuda-graph",
                       "grid": [args.n] * 3, "case_steps": 500, "window": f"steps 1-{K} from rest",
                       "l2": "inputs larger than L2: state is 9 FP64 arrays of "
                             f"{(args.n + 4) ** 3 * 8 / 1e6:.0f} MB, no flush",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "sor_sweeps_total": int(sum(sweeps)), "sor_sweeps_per_step": float(np.mean(sweeps)),
            "sweep_rate": {"value": round(cells_total * float(sum(sweeps)) / (ms_max * 1e-3) / 1e6, 2),
                           "unit": "Mcell-sweeps/s"},
            "all_converged": bool(all(i.converged for i in info)),
            "gpu_launches": launches * world,
            "adjoint_over_forward": adj["mixed"]["adjoint_over_forward"] if adj else None,
            "adjoint": adj,
            "roofline": rl, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        import torch.distributed as dist
        barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ reference arm
def reference_cavity(n, Re, dt):
    """Parameters and grid of the cavity for the reference arm, made without
    the product library: the grid by the oracle's restatement of
    gridder_equal (gridder.f90:228-327), the parameters as a plain struct."""
    from oracle import cpu_oracle
    from ntustcfdlab_b200.abi import SOR_LEX, f4, make_params
    p = make_params(n, n, n, Re=Re, dt=f4(dt), sor_order=SOR_LEX,
                    bc={"North": ("Dirichlet", "no-slip", "no-slip")})
    return p, cpu_oracle.gridder_equal(n, n, n, 1.0, 1.0, 1.0)


def run_reference(args):
    """The CPU restatement of the reference's algorithm (lexicographic SOR,
    the reference's OpenMP loop schedule, every host thread) on the same
    window as our arm: W warm-up steps, a reset to the initial state, then
    steps 1..K from rest, bounded by a time budget.  This process never
    loads the CUDA library."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import cpu_oracle
    p, grid = reference_cavity(args.n, args.Re, args.dt)
    cells = args.n ** 3
    threads = os.cpu_count() or 1
    o = cpu_oracle.Oracle(p, grid, threads=threads)
    o.initial_conditions()
    o.boundary_conditions()
    if args.warmup > 0:
        o.step(args.warmup)
    o.initial_conditions()
    o.boundary_conditions()
    budget = 150.0
    t0 = time.perf_counter()
    done = sweeps = 0
    for _ in range(args.steps):
        inf = o.step(1)[0]
        done += 1
        sweeps += inf.sor_iters
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    value = cells * done / el / 1e6
    sample = (f"steps 1-{done} of the {args.n}^3 cavity from rest after {args.warmup} warm-up steps "
              f"and a reset ({sweeps} SOR sweeps, {el:.1f} s; at most {budget:.0f} s of steps)")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
            "n_gpus": 0, "steps": done, "warmup": args.warmup, "ms_per_step": el * 1e3 / done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (lid-driven cavity from rest, no dataset)",
            "config": {"workload": f"lid-driven cavity {args.n}^3, Re={args.Re:g}, dt={args.dt:g}, zeta=1e-4",
                       "grid": [args.n] * 3, "window": f"steps 1-{done} from rest",
                       "parallelism": f"{threads} OpenMP threads"},
            "sor_sweeps_total": sweeps, "sor_sweeps_per_step": sweeps / done,
            "sweep_rate": {"value": round(cells * sweeps / el / 1e6, 3), "unit": "Mcell-sweeps/s"},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the Fortran/MPI reference cannot be compiled here (no Fortran compiler, no "
                    "MPI); this arm runs the C++ restatement of its algorithm with the reference's "
                    "lexicographic SOR and OpenMP loop schedule, with the grid from the same "
                    "restatement (the CUDA library is not loaded)"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
