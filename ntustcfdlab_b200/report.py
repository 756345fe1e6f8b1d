"""Per-case GPU numbers for the configurations C1-C5: step throughput of the
plain FP64 path and of the mixed path, SOR sweeps per step, relative L2
difference of the mixed state from the FP64 state after the same steps, and
the largest |div u| V of the last step.

    python -m ntustcfdlab_b200.report [--cases c1,c2,c3,c4,c5] [--out report.json]

Each case starts from its own initial state (zero fields, or the uniform
inflow for the cylinder), builds its mask, runs a few untimed steps for the
graph instantiation, resets, and times `steps` steps with the CUDA events of
ntcfd_step.  The big airfoil cases run a fixed window of their first steps,
stated in the output.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import cases
from .abi import FP64, MIXED, params_copy
from .solver import Solver

# case -> (factory, steps timed, mixed_cycle)
WINDOWS = {"c1": (cases.c1, 200), "c2": (cases.c2, 500), "c3": (cases.c3, 50),
           "c4": (cases.c4, 200), "c5": (cases.c5, 10)}


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


def run_case(name: str, cycle: int = 8) -> dict:
    fn, steps = WINDOWS[name]
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
            info, rc = s.step(steps)
            ms = s.last_step_ms()
            states[tag] = s.get_state()
            out[tag] = {"ms_per_step": ms / steps, "mcell_steps_per_s": c.cells * steps / (ms * 1e3),
                        "sweeps_per_step": float(np.mean([i.sor_iters for i in info])),
                        "all_converged": bool(all(i.converged for i in info)),
                        "div_max_last": info[-1].div_max,
                        "sor_path": {1: "streaming", 2: "resident"}.get(info[0].sor_path),
                        "cDrag_last": info[-1].cDrag, "cLift_last": info[-1].cLift}
        finally:
            s.close()
    out["mixed_over_fp64"] = out["mixed"]["mcell_steps_per_s"] / out["fp64"]["mcell_steps_per_s"]
    rel = {}
    for k, a, b in zip("uvwp", states["mixed"], states["fp64"]):
        a, b = a[2:-2, 2:-2, 2:-2], b[2:-2, 2:-2, 2:-2]
        nb = float(np.linalg.norm(b))
        rel[k] = float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a - b))
    out["rel_l2_mixed_vs_fp64"] = rel
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", default="c1,c2,c3,c4,c5")
    ap.add_argument("--cycle", type=int, default=8)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    res = []
    for name in args.cases.split(","):
        r = run_case(name.strip(), args.cycle)
        print(json.dumps(r), flush=True)
        res.append(r)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
