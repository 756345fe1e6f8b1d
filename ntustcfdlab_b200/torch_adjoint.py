"""torch.autograd wrapper of the discrete adjoint (verification harness).

``ForceObjective`` is a ``torch.autograd.Function`` whose forward runs
ntcfd_adjoint over K steps from a fixed initial state and returns the
objective J = mean(w_drag cDrag + w_lift cLift); its backward returns the
adjoint gradients that the same call produced, scaled by the incoming
gradient.  The inputs are the inflow speed U, the inflow angle theta
(radians) and the body force (3, nx, ny, nz); each call builds a fresh
context from ``case_fn(U, theta)`` holding the given initial state (ghosts
included, so it does not depend on U and theta), so
``torch.autograd.gradcheck`` compares the adjoint with central finite
differences of complete K-step runs.

Torch here is only the caller's autograd plumbing: every step and every
adjoint kernel runs through libntcfd.so.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .solver import Solver


def make_solver(case, state=None, apply_bc: bool | None = None) -> Solver:
    """Context for a case: grid, mask from case.mask and a state.  With no
    state the fields are zero and boundary_conditions() sets the ghosts;
    a given state (u, v, w, p halo arrays, ghosts included) is used as it is
    unless apply_bc is true."""
    s = Solver(case.params, case.grid)
    m = case.mask
    if m.get("kind") == "cylinder":
        s.build_mask_cylinder(m["zc"], m["yc"], m["r"])
    elif m.get("kind") == "naca":
        s.build_mask_polygon(m["az"], m["ay"], m["aoa"], m["zc"], m["yc"])
    if state is not None:
        s.set_state(*state)
    if apply_bc or (apply_bc is None and state is None):
        s.boundary_conditions()
    return s


class ForceObjective(torch.autograd.Function):
    """J(U, theta, f) over `nsteps` steps; see the module docstring."""

    @staticmethod
    def forward(ctx, U, theta, force, case_fn, state, nsteps, checkpoint_every, w_drag, w_lift,
                adj_zeta):
        case = case_fn(float(U), float(theta))
        s = make_solver(case, state)
        try:
            f = force.detach().cpu().numpy()
            s.set_body_force(*[np.asfortranarray(f[c]) for c in range(3)])
            r = s.adjoint(nsteps, checkpoint_every, w_drag=w_drag, w_lift=w_lift, adj_zeta=adj_zeta,
                          inflow=("Back", 2, 1))
        finally:
            s.close()
        gf = np.stack([np.asarray(a) for a in r["dJ_df"]])
        ctx.save_for_backward(torch.tensor(r["dJ_dU"], dtype=torch.float64),
                              torch.tensor(r["dJ_dtheta"], dtype=torch.float64),
                              torch.from_numpy(gf))
        return torch.tensor(r["J"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        dU, dth, df = ctx.saved_tensors
        need = ctx.needs_input_grad
        return (gJ * dU if need[0] else None, gJ * dth if need[1] else None,
                gJ * df if need[2] else None) + (None,) * 7


def objective(U, theta, force, case_fn, state, nsteps, checkpoint_every, w_drag=1.0, w_lift=0.0,
              adj_zeta=1e-12):
    return ForceObjective.apply(U, theta, force, case_fn, state, nsteps, checkpoint_every, w_drag,
                                w_lift, adj_zeta)


def inflow_case_fn(base_fn):
    """case_fn(U, theta) from a cylinder_crossflow-style factory taking
    U and theta_deg keywords."""
    def fn(U, theta):
        return base_fn(U=U, theta_deg=math.degrees(theta))
    return fn
