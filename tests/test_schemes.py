"""The uncalled K2 predictors of the reference (discretisation_QUICK.f90,
discretisation_upwind.f90, discretisation_centre.f90) in the oracle: closed
forms that hold whatever the transcription's rounding.

* A uniform stream is a fixed point of all three: every flux difference and
  every diffusion term vanishes.
* On a uniform grid and a velocity field linear in every coordinate, with
  values exactly representable, the QUICK curvature terms are exactly zero
  and QUICK's face values equal the node means, so QUICK and centre predict
  the same u*, v*, w* to the last bit; upwind does not.
* Only i < nx (u), j < ny (v), k < nz (w) are predicted: the wall faces keep
  the u -> u_star copy of boundary_conditions.f90:305-324.
"""
import numpy as np
import pytest

from ntustcfdlab_b200.abi import CENTRE, QUICK, QUICK_CENTRE, UPWIND, make_params

N = (6, 7, 8)


def oracle_for(scheme, les=0):
    from oracle import cpu_oracle
    p = make_params(*N, Re=100.0, dt=0.01, scheme=scheme, LES=les, Cs=0.18)
    o = cpu_oracle.Oracle(p, cpu_oracle.gridder_equal(*N, 3.0, 3.5, 4.0))   # spacing 0.5
    o.initial_conditions()
    return o


def set_fields(o, fu, fv, fw):
    shape = tuple(n + 4 for n in N)
    idx = np.indices(shape) - 1                  # Fortran index -1..n+2
    for name, f in (("u", fu), ("v", fv), ("w", fw)):
        o.set(name, np.asfortranarray(f(*idx).astype(np.float64)))
        o.set(name + "_star", np.asfortranarray(f(*idx).astype(np.float64)))


def predicted(o):
    o.predictor()
    return [o.get(n) for n in ("u_star", "v_star", "w_star")]


@pytest.mark.parametrize("scheme", [QUICK, UPWIND, CENTRE])
@pytest.mark.parametrize("les", [0, 1])
def test_uniform_stream_is_a_fixed_point(scheme, les):
    o = oracle_for(scheme, les)
    set_fields(o, lambda i, j, k: 0 * i + 0.75, lambda i, j, k: 0 * i - 0.25, lambda i, j, k: 0 * i + 1.5)
    us, vs, ws = predicted(o)
    assert np.all(us == 0.75) and np.all(vs == -0.25) and np.all(ws == 1.5)


def test_quick_equals_centre_on_linear_fields():
    fu = lambda i, j, k: 1.0 + 0.5 * i - 0.25 * j + 0.125 * k
    fv = lambda i, j, k: -0.5 + 0.25 * i + 0.5 * j - 0.25 * k
    fw = lambda i, j, k: 2.0 - 0.125 * i + 0.25 * j + 0.5 * k
    out = {}
    for scheme in (QUICK, CENTRE, UPWIND):
        o = oracle_for(scheme)
        set_fields(o, fu, fv, fw)
        out[scheme] = predicted(o)
    inner = np.s_[2:-2, 2:-2, 2:-2]
    for a, b in zip(out[QUICK], out[CENTRE]):
        assert np.array_equal(a[inner], b[inner])
    assert not np.array_equal(out[UPWIND][0][inner], out[CENTRE][0][inner])


@pytest.mark.parametrize("scheme", [QUICK, UPWIND, CENTRE])
def test_wall_faces_are_not_predicted(scheme):
    rng = np.random.default_rng(4)
    shape = tuple(n + 4 for n in N)
    fields = [rng.standard_normal(shape) for _ in range(3)]
    o = oracle_for(scheme)
    for name, a in zip("uvw", fields):
        o.set(name, np.asfortranarray(a))
        o.set(name + "_star", np.asfortranarray(a))
    us, vs, ws = predicted(o)
    nx, ny, nz = N
    # array index = Fortran index + 1
    assert np.array_equal(us[nx + 1, 2:ny + 2, 2:nz + 2], fields[0][nx + 1, 2:ny + 2, 2:nz + 2])
    assert np.array_equal(vs[2:nx + 2, ny + 1, 2:nz + 2], fields[1][2:nx + 2, ny + 1, 2:nz + 2])
    assert np.array_equal(ws[2:nx + 2, 2:ny + 2, nz + 1], fields[2][2:nx + 2, 2:ny + 2, nz + 1])
    assert not np.array_equal(us[nx, 2:ny + 2, 2:nz + 2], fields[0][nx, 2:ny + 2, 2:nz + 2])
    # QUICK_centre predicts the wall faces too (Q4)
    o = oracle_for(QUICK_CENTRE)
    for name, a in zip("uvw", fields):
        o.set(name, np.asfortranarray(a))
    o.smagorinsky()
    us2 = predicted(o)[0]
    assert not np.array_equal(us2[nx + 1, 2:ny + 2, 2:nz + 2], fields[0][nx + 1, 2:ny + 2, 2:nz + 2])


@pytest.mark.parametrize("sign", [1.0, -1.0])
@pytest.mark.parametrize("axis", [0, 1, 2])
def test_quick_is_exact_on_quadratics(axis, sign):
    """QUICK face values reproduce a quadratic exactly, in either branch.  One
    component varies quadratically along its own axis, the others are zero,
    so its prediction is the 1-D closed form
        f* = f - dt (F(a+1/2)^2 - F(a-1/2)^2) / h + nu dt (f(a+1) - 2 f(a) + f(a-1)) / h^2.
    Spacing 0.5, dt = 1/8, nu = 1/128 and the dyadic values make every
    operation exact, so the comparison is bitwise."""
    from oracle import cpu_oracle
    h, dt, Re = 0.5, 0.125, 128.0
    p = make_params(*N, Re=Re, dt=dt, scheme=QUICK)
    o = cpu_oracle.Oracle(p, cpu_oracle.gridder_equal(*N, N[0] * h, N[1] * h, N[2] * h))
    o.initial_conditions()
    q = lambda a: sign * (0.25 * a * a + 0.5)
    zero = lambda i, j, k: 0.0 * i
    f = lambda i, j, k: q((i, j, k)[axis])
    fs = [zero, zero, zero]
    fs[axis] = f
    set_fields(o, *fs)
    got = predicted(o)[axis]
    idx = np.indices(got.shape) - 1
    a = idx[axis].astype(np.float64)
    want = q(a) - dt * (q(a + 0.5) ** 2 - q(a - 0.5) ** 2) / h + (1.0 / Re) * dt * (q(a + 1) - 2 * q(a) + q(a - 1)) / h ** 2
    lo = [2, 2, 2]
    hi = [n + 2 for n in N]
    hi[axis] -= 1                       # the wall face is not predicted
    sl = tuple(slice(l, u) for l, u in zip(lo, hi))
    assert np.array_equal(got[sl], want[sl])


@pytest.mark.parametrize("sign", [1.0, -1.0])
def test_upwind_takes_the_upstream_node(sign):
    """discretisation_upwind.f90 on u = sign (1 + i/2) along x, v = w = 0:
    the face-averaged velocities all have the sign of u, so both x faces
    take the node on the upstream side."""
    from oracle import cpu_oracle
    h, dt, Re = 0.5, 0.125, 128.0
    p = make_params(*N, Re=Re, dt=dt, scheme=UPWIND)
    o = cpu_oracle.Oracle(p, cpu_oracle.gridder_equal(*N, N[0] * h, N[1] * h, N[2] * h))
    o.initial_conditions()
    g = lambda a: sign * (1.0 + 0.5 * a)
    set_fields(o, lambda i, j, k: g(i), lambda i, j, k: 0.0 * i, lambda i, j, k: 0.0 * i)
    got = predicted(o)[0]
    a = (np.indices(got.shape) - 1)[0].astype(np.float64)
    ut1, ut2 = 0.5 * (g(a) + g(a + 1)), 0.5 * (g(a - 1) + g(a))
    ue = g(a) if sign > 0 else g(a + 1)
    uw = g(a - 1) if sign > 0 else g(a)
    want = g(a) - dt * (ut1 * ue - ut2 * uw) / h       # linear u: no diffusion
    sl = np.s_[2:N[0] + 1, 2:-2, 2:-2]
    assert np.array_equal(got[sl], want[sl])
