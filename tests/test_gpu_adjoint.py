"""Discrete adjoint (ntcfd_adjoint) against central finite differences of
complete K-step runs, against itself under other checkpoint spacings, SOR
paths and precisions, and through the torch.autograd harness.

Set-up: a cylinder in cross-flow on 8 x 24 x 32 cells, inflow at 5 degrees,
off-centre body, started from a seeded perturbed uniform flow so that no
QUICK advecting velocity is exactly zero.  The forward pressure solves run
to zeta = 1e-12 so that h = 1e-6 differences resolve the derivative.
"""
import math

import numpy as np
import pytest

from ntustcfdlab_b200 import abi, cases
from ntustcfdlab_b200.solver import Solver

pytestmark = pytest.mark.gpu

K = 6          # steps of the objective
H = 1e-6       # central-difference step
FD_RTOL = 1e-4
W_DRAG, W_LIFT = 1.0, 0.5


def small_case(U=1.0, theta_deg=5.0, precision=abi.FP64, LES=0, sor_path=abi.SOR_AUTO):
    kw = dict(zeta=1e-12, itmax=200000, sor_path=sor_path)
    if precision == abi.MIXED:
        kw["mixed_cycle"] = 8
    if LES:
        kw.update(LES=1, Cs=abi.f4(0.18))
    return cases.cylinder_crossflow(8, 24, 32, 1.0, 6.0, 8.0, zc=2.55, yc=3.1, D=1.0, Re=100.0,
                                    dt=0.01, U=U, theta_deg=theta_deg, steps=K,
                                    precision=precision, **kw)


def raw_state(case, seed=7):
    p = case.params
    shape = (p.nx + 4, p.ny + 4, p.nz + 4)
    rng = np.random.default_rng(seed)
    th = math.radians(5.0)
    u = 0.05 * rng.standard_normal(shape)
    v = math.sin(th) + 0.05 * rng.standard_normal(shape)
    w = math.cos(th) + 0.05 * rng.standard_normal(shape)
    return tuple(np.asfortranarray(a) for a in (u, v, w, np.zeros(shape)))


def initial_state(case, seed=7):
    """The seeded state with the ghosts of the base case's boundary
    conditions: fixed, whatever inflow a run is given."""
    s = Solver(case.params, case.grid)
    try:
        s.set_state(*raw_state(case, seed))
        s.boundary_conditions()
        return s.get_state()
    finally:
        s.close()


def solver_for(case, state, force=None, apply_bc=False):
    from ntustcfdlab_b200.torch_adjoint import make_solver
    s = make_solver(case, state, apply_bc=apply_bc)
    if force is not None:
        s.set_body_force(*force)
    return s


def objective(case, state, force=None, apply_bc=False):
    s = solver_for(case, state, force, apply_bc)
    try:
        info, rc = s.step(K)
        assert rc == 0
        return sum(W_DRAG * i.cDrag + W_LIFT * i.cLift for i in info) / K
    finally:
        s.close()


def run_adjoint(case, state, force=None, M=2, **kw):
    s = solver_for(case, state, force)
    try:
        r = s.adjoint(K, M, w_drag=W_DRAG, w_lift=W_LIFT, adj_zeta=1e-12, inflow=("Back", 2, 1), **kw)
        assert r["status"] == 0, r
        r["state"] = s.get_state()
        return r
    finally:
        s.close()


@pytest.fixture(scope="module")
def base():
    case = small_case()
    state = initial_state(case)
    force = cases.body_force_c4((case.params.nx, case.params.ny, case.params.nz), scale=1e-2)
    return case, state, force, run_adjoint(case, state, force)


def test_objective_matches_plain_steps(base):
    case, state, force, r = base
    assert r["J"] == objective(case, state, force)


def test_state_after_adjoint_equals_plain_steps(base):
    case, state, force, r = base
    s = solver_for(case, state, force)
    try:
        s.step(K)
        ref = s.get_state()
    finally:
        s.close()
    for a, b in zip(r["state"], ref):
        assert np.array_equal(a, b)


def _fd(fn, x, h=H):
    return (fn(x + h) - fn(x - h)) / (2 * h)


def test_inflow_speed_and_angle_match_central_differences(base):
    case, state, force, r = base
    th0 = 5.0
    gU = _fd(lambda U: objective(small_case(U=U, theta_deg=th0), state, force), 1.0)
    gth = _fd(lambda t: objective(small_case(theta_deg=math.degrees(t)), state, force), math.radians(th0))
    assert abs(r["dJ_dU"] - gU) <= FD_RTOL * abs(gU), (r["dJ_dU"], gU)
    assert abs(r["dJ_dtheta"] - gth) <= FD_RTOL * abs(gth), (r["dJ_dtheta"], gth)


def test_dirichlet_value_gradient_matches_central_differences(base):
    # the tangential inflow value alone (bc_value[Back][v])
    case, state, force, r = base

    def J(val):
        c = small_case()
        c.params.bc_value[4][1] = val
        return objective(c, state, force)

    v0 = case.params.bc_value[4][1]
    g = _fd(J, v0)
    assert abs(r["dJ_dbc"][4, 1] - g) <= FD_RTOL * abs(g), (r["dJ_dbc"][4, 1], g)


def test_body_force_directional_derivative(base):
    case, state, force, r = base
    rng = np.random.default_rng(11)
    d = [np.asfortranarray(rng.standard_normal(f.shape)) for f in force]
    g = _fd(lambda h: objective(case, state, [f + h * e for f, e in zip(force, d)]), 0.0)
    ga = sum(float(np.sum(a * e)) for a, e in zip(r["dJ_df"], d))
    assert abs(ga - g) <= FD_RTOL * abs(g), (ga, g)


def _rel(qs, rs):
    num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(qs, rs))
    den = sum(float(np.sum(b ** 2)) for b in rs)
    return math.sqrt(num / den)


def test_gradients_do_not_depend_on_checkpoint_spacing(base):
    # recomputed states are bit-identical; the adjoint's scatter atomics are
    # not ordered, so the gradients agree to rounding
    case, state, force, r = base
    for M in (1, 4, K):
        q = run_adjoint(case, state, force, M=M)
        nck = (K + M - 1) // M
        assert q["recomputed_steps"] == (K - nck) - (K - (nck - 1) * M - 1)
        assert np.allclose(q["dJ_dbc"], r["dJ_dbc"], rtol=1e-10, atol=1e-14)
        assert _rel(q["dJ_df"], r["dJ_df"]) <= 1e-10


def test_streaming_and_resident_sor_give_the_same_adjoint(base):
    case, state, force, r = base
    q = run_adjoint(small_case(sor_path=abi.SOR_STREAMING), state, force)
    assert abs(q["dJ_dU"] - r["dJ_dU"]) <= 1e-9 * abs(r["dJ_dU"])
    assert _rel(q["dJ_df"], r["dJ_df"]) <= 1e-9


def test_mixed_precision_adjoint_matches_fp64(base):
    case, state, force, r = base
    q = run_adjoint(small_case(precision=abi.MIXED), state, force)
    assert abs(q["dJ_dU"] - r["dJ_dU"]) <= 1e-6 * abs(r["dJ_dU"])
    assert abs(q["dJ_dtheta"] - r["dJ_dtheta"]) <= 1e-6 * abs(r["dJ_dtheta"])
    assert _rel(q["dJ_df"], r["dJ_df"]) <= 1e-6


def test_initial_boundary_conditions_are_differentiated():
    # the state's ghosts set by the run's own inflow values (as main.f90:100 does)
    case = small_case()
    raw = raw_state(case)
    s = solver_for(case, raw)
    try:
        r = s.adjoint(K, 2, w_drag=W_DRAG, w_lift=W_LIFT, adj_zeta=1e-12, inflow=("Back", 2, 1),
                      initial_bc=True, force_grad=False)
    finally:
        s.close()
    assert r["J"] == objective(case, raw, apply_bc=True)
    gU = _fd(lambda U: objective(small_case(U=U), raw, apply_bc=True), 1.0)
    assert abs(r["dJ_dU"] - gU) <= FD_RTOL * abs(gU), (r["dJ_dU"], gU)


def test_les_adjoint_matches_central_differences():
    case = small_case(LES=1)
    state = initial_state(case)
    r = run_adjoint(case, state)
    gU = _fd(lambda U: objective(small_case(U=U, LES=1), state), 1.0)
    assert abs(r["dJ_dU"] - gU) <= FD_RTOL * abs(gU), (r["dJ_dU"], gU)


def test_torch_gradcheck_on_inflow():
    torch = pytest.importorskip("torch")
    from ntustcfdlab_b200.torch_adjoint import objective as tobj

    case0 = small_case()
    state = initial_state(case0)
    force = torch.zeros((3, 8, 24, 32), dtype=torch.float64)

    def case_fn(U, theta):
        return small_case(U=U, theta_deg=math.degrees(theta))

    def f(U, th):
        return tobj(U, th, force, case_fn, state, K, 2, W_DRAG, W_LIFT)

    U = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    th = torch.tensor(math.radians(5.0), dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(f, (U, th), eps=H, atol=1e-7, rtol=FD_RTOL)


# ---------------------------------------------------------------- body angle
AOA_B, ZC_B, YC_B, WIDTH = 8.0, 2.3, 3.1, 0.3


def _smooth_solver(case, state, aoa):
    from ntustcfdlab_b200.solver import naca4_polygon
    z, y = naca4_polygon(0.12, 64)
    s = Solver(case.params, case.grid)
    s.set_state(*state)
    s.build_mask_smooth(z, y, aoa, ZC_B, YC_B, WIDTH)
    return s


def _smooth_objective(case, state, aoa):
    s = _smooth_solver(case, state, aoa)
    try:
        info, rc = s.step(K)
        assert rc == 0
        J = 0.0                         # summed in the adjoint's order (sum() compensates)
        for i in info:
            J += W_DRAG * i.cDrag + W_LIFT * i.cLift
        return J / K
    finally:
        s.close()


def test_body_angle_gradient_matches_central_differences():
    """dJ/dAOA through the rotating body (the smoothed NACA0012 mask of
    ntcfd_build_mask_smooth), against central differences of complete K-step
    runs with the same mask at AOA +- h; beside it the freestream-angle
    gradient of the same run, a different quantity."""
    case = small_case()
    state = initial_state(case)
    s = _smooth_solver(case, state, AOA_B)
    try:
        eta = s.get_mask()
        # a 12 % thick section on 0.25 cells, blurred over +-0.3: no cell is fully inside
        assert eta.min() >= 0.0 and 0.5 < eta.max() <= 1.0
        assert np.count_nonzero((eta > 0) & (eta < 1)) > 50          # the blurred band
        r = s.adjoint(K, 2, w_drag=W_DRAG, w_lift=W_LIFT, adj_zeta=1e-12, inflow=("Back", 2, 1))
        assert r["status"] == 0
    finally:
        s.close()
    assert r["J"] == _smooth_objective(case, state, AOA_B)
    h = 1e-4                                                         # degrees
    g = (_smooth_objective(case, state, AOA_B + h) - _smooth_objective(case, state, AOA_B - h)) / (2 * h)
    g *= 180.0 / math.pi                                             # per radian
    assert abs(g) > 1e-3
    assert abs(r["dJ_daoa_body"] - g) <= FD_RTOL * abs(g), (r["dJ_daoa_body"], g)
    assert r["dJ_daoa_body"] != r["dJ_dtheta"]


def test_body_angle_gradient_is_zero_without_the_smoothed_mask(base):
    case, state, force, r = base
    assert r["dJ_daoa_body"] == 0.0
