"""Dynamic angle of attack (dynamic_AOA + RayCasting every step,
airfoil.f90:311-321, main.f90:144-155) against the oracle stepping with the
same angles, and the asynchronous centred output."""
import math

import numpy as np
import pytest

from conftest import interior, rel_l2
from ntustcfdlab_b200 import abi
from ntustcfdlab_b200.abi import NtcfdStepInfo, dptr, f4, make_params, params_copy

pytestmark = pytest.mark.gpu

N = (4, 48, 64)
L = (1.0, 3.0, 4.0)
BAND = (f4(12.5), 1.5, 1.2, 4, 20, 30, 24, 36, 1.0, f4(0.3), f4(0.6), f4(1.1), 2.0)
AOA1, RF, ZC, YC, START, STEPS = 5.0, 2.0, 1.2, 1.5, 2, 4


def params():
    bc = {"West": ("periodic",) * 3, "East": ("periodic",) * 3,
          "South": ("Neumann",) * 3, "North": ("Neumann",) * 3,
          "Back": ("Dirichlet", "Dirichlet", "Dirichlet"), "Front": ("Neumann",) * 3}
    return make_params(*N, Re=1000.0, dt=f4(1e-3), bc=bc, bc_value={"Back": (0.0, 0.0, 1.0)}, lx=L[0])


def dynamic_aoa(t, dt, start=START):
    # airfoil.f90:313-317 with the default-real PI literal
    pi = float(np.float32(3.14159265359))
    frequency = RF / pi
    return AOA1 + 10 * abs(math.sin(2 * pi * frequency * (t - dt * (start - 1))))


# the moving-body graph (mask kernels, then the step under an IF node) around
# the resident and the streaming solve, and the eager launches
PATHS = [dict(), dict(sor_path=abi.SOR_STREAMING), dict(eager=1)]


@pytest.mark.parametrize("path", PATHS, ids=["graph-resident", "graph-streaming", "eager"])
def test_dynamic_angle_matches_oracle(orc, path):
    from ntustcfdlab_b200.solver import Solver, gridder_unequal, naca4_polygon
    z, y = naca4_polygon(0.12, 64)
    grid = gridder_unequal(*N, *L, BAND)
    p = params()
    for k, v in path.items():
        setattr(p, k, v)
    # device
    s = Solver(p, grid)
    try:
        s.build_mask_polygon(z, y, AOA1, ZC, YC)          # main.f90:109-110
        s.set_dynamic_aoa(z, y, AOA1, RF, ZC, YC, START)
        s.boundary_conditions()
        info, rc = s.step(STEPS)
        state, eta = s.get_state(), s.get_mask()
    finally:
        s.close()
    # oracle
    og = orc.gridder_unequal(*N, *L, BAND)
    o = orc.Oracle(p, og)
    o.initial_conditions()
    assert o.raycasting(z, y, AOA1, ZC, YC) == 0
    o.boundary_conditions()
    angles, oi = [], []
    for istep in range(1, STEPS + 1):
        a = 0.0
        if istep >= START:
            a = dynamic_aoa(o.time, p.dt)
            assert o.raycasting(z, y, a, ZC, YC) == 0
        angles.append(a)
        oi += o.step(1)
    assert [i.aoa for i in info] == angles
    assert angles[-1] != angles[-2] != AOA1
    assert np.array_equal(eta, o.get("ETA"))
    assert [i.sor_iters for i in info] == [i.sor_iters for i in oi]
    for k, a in zip("uvwp", state):
        assert rel_l2(interior(a), interior(o.get(k))) <= 1e-12, k


@pytest.mark.parametrize("eager", [0, 1])
def test_a_tie_stops_the_call_after_the_steps_before_it(eager):
    """A body whose pivot vertex (0.25, 0) sits on a grid node ties at every
    angle: the call runs the steps before start_step, then stops with
    NTCFD_EINVAL.  The time, the step count and the records count exactly
    those steps, ETA holds the tied step's mask (as the allocation-free
    builder makes it at that angle), and the next call stops at once."""
    import ctypes
    from ntustcfdlab_b200.solver import Solver, gridder_equal
    n, zc, yc, start = (3, 32, 32), 1.0, 2.0, 3
    p = make_params(*n, Re=100.0, dt=f4(1e-3), eager=eager)
    s = Solver(p, gridder_equal(*n, 1.0, 4.0, 4.0))
    z = np.ascontiguousarray([0.25, 0.61, 1.03, 0.58, 0.25])
    y = np.ascontiguousarray([0.0, 0.37, 0.013, -0.33, 0.0])
    try:
        s.set_dynamic_aoa(z, y, AOA1, RF, zc, yc, start)
        s.boundary_conditions()
        info = (NtcfdStepInfo * 5)()
        assert s.lib.ntcfd_step(s.h, 5, info) == abi.NTCFD_EINVAL
        assert "(2 ran)" in s._err() and "ties" in s._err(), s._err()
        t = 0.0
        for _ in range(2):
            t = t + p.dt
        assert s.time == t
        assert info[0].sor_iters > 0 and info[1].sor_iters > 0 and info[2].sor_iters == 0
        eta = s.get_mask()
        assert eta.any()
        ties = ctypes.c_int(-1)
        assert s.lib.ntcfd_build_mask_polygon_noalloc(s.h, dptr(z), dptr(y), len(z), dynamic_aoa(t, p.dt, start),
                                                      zc, yc, ctypes.byref(ties)) == abi.NTCFD_EINVAL
        assert ties.value > 0
        np.testing.assert_array_equal(s.get_mask(), eta)
        assert s.lib.ntcfd_step(s.h, 1, info) == abi.NTCFD_EINVAL
        assert "(0 ran)" in s._err()
        assert s.time == t
        s.set_dynamic_aoa(None, None, 0, 0, 0, 0, 0)
        info2, rc = s.step(1)
        assert rc == 0 and info2[0].converged and s.time == t + p.dt
    finally:
        s.close()


def test_adjoint_refuses_a_moving_mask():
    from ntustcfdlab_b200.solver import NtcfdError, Solver, gridder_unequal, naca4_polygon
    z, y = naca4_polygon(0.12, 64)
    s = Solver(params(), gridder_unequal(*N, *L, BAND))
    try:
        s.set_dynamic_aoa(z, y, AOA1, RF, ZC, YC, START)
        with pytest.raises(NtcfdError):
            s.adjoint(2, 1)
        s.set_dynamic_aoa(None, None, 0, 0, 0, 0, 0)       # off again
        s.boundary_conditions()
        s.step(1)
    finally:
        s.close()


@pytest.mark.parametrize("pinned", [False, True])
def test_async_output_equals_get_output(pinned):
    import torch
    from ntustcfdlab_b200 import cases
    from ntustcfdlab_b200.solver import NtcfdError, Solver
    c = cases.cavity(24, 100.0, 1e-3, 10)
    s = Solver(c.params, c.grid)

    def buffers():
        if not pinned:     # pageable: staged, then scattered by the stream callback
            return [np.full(s.inner_shape, -1.0, order="F") for _ in range(4)]
        n = int(np.prod(s.inner_shape))
        return [torch.full((n,), -1.0, dtype=torch.float64, pin_memory=True).numpy()
                .reshape(s.inner_shape, order="F") for _ in range(4)]
    try:
        s.boundary_conditions()
        with pytest.raises(NtcfdError):
            s.output_wait()                                  # nothing in flight
        s.step(3)
        s.output_async(buffers())
        ref = s.get_output()
        s.step(2)                                            # overlaps the copy
        got = s.output_wait()
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
        ref = s.get_output()
        first = buffers()
        s.output_async(first)
        s.output_async(buffers())                            # waits for the first
        for a, b in zip(first, ref):
            assert np.array_equal(a, b)
        got2 = s.output_wait()
        for a, b in zip(got2, ref):
            assert np.array_equal(a, b)
        some = buffers()                                     # NULL fields are skipped
        assert s.lib.ntcfd_output_async(s.h, dptr(some[0]), None, None, dptr(some[3])) == 0
        assert s.lib.ntcfd_output_wait(s.h) == 0
        assert np.array_equal(some[0], ref[0]) and np.array_equal(some[3], ref[3])
        assert np.all(some[1] == -1.0) and np.all(some[2] == -1.0)
    finally:
        s.close()
