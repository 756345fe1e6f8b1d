"""Per-case GPU numbers for the configurations C1-C5: step throughput of the
plain FP64 path and of the mixed path, SOR sweeps per step, relative L2
difference of the mixed state from the FP64 state after the same steps, and
the largest |div u| V of the last step.

    python -m ntustcfdlab_b200.report [--cases c1,c2,c3,c4,c5] [--steps N] [--adjoint K] [--out f.json]

Each case starts from its own initial state (zero fields, or the uniform
inflow for the cylinder), builds its mask, runs two untimed steps for the
graph instantiation, resets, and runs its configured number of steps (C1 200,
C2 500, C3 1000, C4 200, C5 2000) timed with the CUDA events of ntcfd_step, in
both precisions.  It reports the fraction of steps whose SOR solve converged
before itmax, the divergence norm and, for C5 with --adjoint K, the adjoint of
the mean lift coefficient over the last K steps.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import cases
from .abi import FP64, MIXED, params_copy
from .solver import Solver

# case -> (factory, steps of the configuration)
WINDOWS = {"c1": (cases.c1, 200), "c2": (cases.c2, 500), "c3": (cases.c3, 1000),
           "c4": (cases.c4, 200), "c5": (cases.c5, 2000)}
CHUNK = 100   # steps per ntcfd_step call


def _initial_state(case):
    if case.mask.get("kind") == "cylinder":
        return cases.uniform_inflow_state(case)
    p = case.params
    z = np.zeros((p.nx + 4, p.ny + 4, p.nz + 4), order="F")
    return (z, z, z, z)


def _solver(case):
    s = Solver(case.params, case.grid)
    m = case.mask
    if m.get("kind") == "cylinder":
        s.build_mask_cylinder(m["zc"], m["yc"], m["r"])
    elif m.get("kind") == "naca":
        s.build_mask_polygon(m["az"], m["ay"], m["aoa"], m["zc"], m["yc"])
    return s


def _device_used_gb():
    try:
        import torch
        free, total = torch.cuda.mem_get_info()
        return (total - free) / 1e9
    except Exception:
        return None


def run_case(name: str, cycle: int = 8, steps: int | None = None, adjoint_K: int = 0, M: int = 25,
             log=print, adj_omega: float = 0.0) -> dict:
    """Both precisions over the case's steps from its initial state (after two
    untimed steps for the graph instantiation and a reset).  With adjoint_K, the
    mixed run saves its state K steps before the end and, after the run, the
    discrete adjoint of the mean cLift over those K steps is taken from it
    (checkpoints every M steps), with respect to the inflow direction of the
    Back wall (normal w, tangential v) and its speed."""
    fn, default_steps = WINDOWS[name]
    steps = steps or default_steps
    out = {"case": name, "steps": steps}
    states = {}
    for prec, tag in ((FP64, "fp64"), (MIXED, "mixed")):
        c = fn(precision=prec)
        c.params = params_copy(c.params, mixed_cycle=cycle if prec == MIXED else 0, diag_divergence=1)
        out["cells"] = c.cells
        out["description"] = c.description
        s = _solver(c)
        try:
            st0 = _initial_state(c)
            s.set_state(*st0)
            s.boundary_conditions()
            s.step(2)                       # graph instantiation, outside the timed steps
            s.set_state(*st0)
            s.boundary_conditions()
            info, ms, saved = [], 0.0, None
            done = 0
            while done < steps:
                if adjoint_K and prec == MIXED and done == steps - adjoint_K:
                    saved = s.get_state()
                n = min(CHUNK, steps - done)
                if adjoint_K and prec == MIXED and done < steps - adjoint_K:
                    n = min(n, steps - adjoint_K - done)
                inf, rc = s.step(n)
                info += inf
                ms += s.last_step_ms()
                done += n
                if done % 500 == 0 or done == steps:
                    log(f"  {name} {tag}: {done}/{steps} steps, {ms / done:.3f} ms/step, "
                        f"sweeps {inf[-1].sor_iters}, converged {inf[-1].converged}")
            states[tag] = s.get_state()
            sw = np.array([i.sor_iters for i in info])
            conv = np.array([i.converged for i in info])
            out[tag] = {"ms_per_step": ms / steps, "mcell_steps_per_s": c.cells * steps / (ms * 1e3),
                        "sweeps_per_step": float(sw.mean()),
                        "sweeps_first10": float(sw[:10].mean()), "sweeps_last100": float(sw[-100:].mean()),
                        "converged_fraction": float(conv.mean()),
                        "first_converged_step": int(np.argmax(conv)) + 1 if conv.any() else None,
                        "all_converged": bool(conv.all()),
                        "div_max_last": info[-1].div_max, "div_max_max": float(max(i.div_max for i in info)),
                        "sor_path": {1: "streaming", 2: "resident"}.get(info[0].sor_path),
                        "cDrag_last": info[-1].cDrag, "cLift_last": info[-1].cLift}
            if prec == MIXED:
                kt = s.time_kernels(10)
                out[tag]["kernel_ms"] = {k: round(v, 5) for k, v in kt.items()}
            if saved is not None:
                s.set_state(*saved)
                r = s.adjoint(adjoint_K, M, w_drag=0.0, w_lift=1.0, inflow=("Back", 2, 1), force_grad=False,
                              adj_itmax=3000, adj_omega=adj_omega)
                out["adjoint"] = {"K": adjoint_K, "M": M, "adj_omega": adj_omega or 1.9,
                                  "objective": "mean cLift over the last K steps",
                                  "J": r["J"], "dJ_dtheta_inflow": r["dJ_dtheta"], "dJ_dU": r["dJ_dU"],
                                  "total_ms": r["total_ms"], "forward_ms": r["forward_ms"],
                                  "recompute_ms": r["recompute_ms"], "solve_ms": r["solve_ms"],
                                  "adjoint_over_forward": r["total_ms"] / r["forward_ms"],
                                  "adj_sweeps": r["adj_sweeps"], "adj_unconverged": r["adj_unconverged"],
                                  "adj_itmax": 3000,
                                  "device_used_gb_after": _device_used_gb()}
                log(f"  {name} adjoint: {out['adjoint']}")
                m = c.mask
                if m.get("kind") == "naca":
                    # the same K steps with the body blurred over +-1.5 cells of the finest
                    # spacing (the smoothed mask is differentiable in the body's angle):
                    # dJ/dAOA through the rotating body beside the freestream angle
                    width = 1.5 * min(float(np.min(c.grid["Dys"][2:-2])), float(np.min(c.grid["Dzs"][2:-2])))
                    s.set_state(*saved)
                    s.build_mask_smooth(m["az"], m["ay"], m["aoa"], m["zc"], m["yc"], width)
                    rb = s.adjoint(adjoint_K, M, w_drag=0.0, w_lift=1.0, inflow=("Back", 2, 1), force_grad=False,
                                   adj_itmax=3000, adj_omega=adj_omega)
                    out["adjoint_body"] = {"K": adjoint_K, "M": M, "mask": f"smoothed, width {width:.5f}",
                                           "J": rb["J"], "dJ_daoa_body_per_rad": rb["dJ_daoa_body"],
                                           "dJ_dtheta_inflow": rb["dJ_dtheta"], "total_ms": rb["total_ms"],
                                           "adjoint_over_forward": rb["total_ms"] / rb["forward_ms"],
                                           "adj_unconverged": rb["adj_unconverged"],
                                           "device_used_gb_after": _device_used_gb()}
                    log(f"  {name} adjoint through the body: {out['adjoint_body']}")
        finally:
            s.close()
    out["mixed_over_fp64"] = out["mixed"]["mcell_steps_per_s"] / out["fp64"]["mcell_steps_per_s"]
    rel = {}
    for k, a, b in zip("uvwp", states["mixed"], states["fp64"]):
        a, b = a[2:-2, 2:-2, 2:-2], b[2:-2, 2:-2, 2:-2]
        nb = float(np.linalg.norm(b))
        rel[k] = float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a - b))
    out["rel_l2_mixed_vs_fp64"] = rel
    # the velocity as one vector field: a component that is nearly zero everywhere
    # (the span velocity of a 2-D flow) has a large relative error of no weight
    num = sum(float(np.linalg.norm(a[2:-2, 2:-2, 2:-2] - b[2:-2, 2:-2, 2:-2])) ** 2
              for a, b in zip(states["mixed"][:3], states["fp64"][:3]))
    den = sum(float(np.linalg.norm(b[2:-2, 2:-2, 2:-2])) ** 2 for b in states["fp64"][:3])
    out["rel_l2_velocity_mixed_vs_fp64"] = (num / den) ** 0.5 if den > 0 else num ** 0.5
    out["norm_fp64"] = {k: float(np.linalg.norm(b[2:-2, 2:-2, 2:-2])) for k, b in zip("uvwp", states["fp64"])}
    return out


def moving_body_cost(name: str = "c3", steps: int = 200, rf: float = 2.0, log=print) -> dict:
    """Per-step cost of a moving body (ntcfd_set_dynamic_aoa) on an airfoil
    case, mixed precision, from the case's initial state.  Three runs of the
    same steps: the static mask; the mask rebuilt every step at the same angle
    (reduced frequency 0: identical flow and sweeps, so the difference is the
    mask kernels alone); and a pitching body (reduced frequency rf).  Two
    untimed steps come first in each (the pitching angles start two steps in)."""
    fn, _ = WINDOWS[name]
    out = {"case": name, "steps": steps, "reduce_frequency": rf}
    for tag, f in (("static", None), ("rebuilt_same_angle", 0.0), ("pitching", rf)):
        c = fn(precision=MIXED)
        m = c.mask
        s = _solver(c)
        try:
            st0 = _initial_state(c)
            if f is not None:
                s.set_dynamic_aoa(m["az"], m["ay"], m["aoa"], f, m["zc"], m["yc"], 1)
            s.set_state(*st0)
            s.boundary_conditions()
            s.step(2)                       # graph instantiation, outside the timed steps
            s.set_state(*st0)
            s.boundary_conditions()
            info, ms, done = [], 0.0, 0
            while done < steps:
                n = min(CHUNK, steps - done)
                inf, rc = s.step(n)
                info += inf
                ms += s.last_step_ms()
                done += n
            sw = np.array([i.sor_iters for i in info])
            out[tag] = {"ms_per_step": ms / steps, "sweeps_per_step": float(sw.mean()),
                        "launches_per_step": float(np.mean([i.launches for i in info])),
                        "aoa_min": float(min(i.aoa for i in info)), "aoa_max": float(max(i.aoa for i in info)),
                        "cLift_last": info[-1].cLift}
            log(f"  {name} {tag}: {out[tag]}")
        finally:
            s.close()
    st, same = out["static"], out["rebuilt_same_angle"]
    out["mask_ms_per_step"] = same["ms_per_step"] - st["ms_per_step"]
    out["same_sweeps"] = st["sweeps_per_step"] == same["sweeps_per_step"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", default="c1,c2,c3,c4,c5")
    ap.add_argument("--cycle", type=int, default=8)
    ap.add_argument("--steps", type=int, default=None, help="override the configured step count")
    ap.add_argument("--adjoint", type=int, default=0, help="C5: adjoint of mean cLift over the last K steps")
    ap.add_argument("--out", default=None)
    ap.add_argument("--adj-omega", type=float, default=0.0,
                    help="SOR relaxation of the C5 adjoint solves (0: the library's 1.9); the best factor "
                         "grows with the grid: 1.9 on C4, about 1.97 on C5")
    ap.add_argument("--moving", type=int, default=0,
                    help="instead: per-step cost of a moving body on c3 over this many steps")
    ap.add_argument("--kernel-times", default=None, metavar="CASE",
                    help="instead: one mixed step of CASE from its initial state, then the "
                         "standalone kernel times (ntcfd_time_kernels, 10 launches each)")
    args = ap.parse_args()
    if args.kernel_times:
        fn, _ = WINDOWS[args.kernel_times]
        c = fn(precision=MIXED)
        s = _solver(c)
        try:
            s.set_state(*_initial_state(c))
            s.boundary_conditions()
            s.step(1)
            kt = s.time_kernels(10)
        finally:
            s.close()
        print(json.dumps({"case": args.kernel_times, "kernel_ms": {k: round(v, 5) for k, v in kt.items()}}))
        return
    if args.moving:
        r = moving_body_cost("c3", args.moving, log=lambda m: print(m, flush=True))
        print(json.dumps(r), flush=True)
        if args.out:
            with open(args.out, "w") as f:
                json.dump(r, f, indent=1)
        return
    res = []
    for name in args.cases.split(","):
        name = name.strip()
        r = run_case(name, args.cycle, args.steps, args.adjoint if name == "c5" else 0,
                     log=lambda m: print(m, flush=True), adj_omega=args.adj_omega)
        print(json.dumps(r), flush=True)
        res.append(r)
        if args.out:
            with open(args.out, "w") as f:
                json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
