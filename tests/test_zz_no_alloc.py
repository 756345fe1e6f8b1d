"""The allocation-free ray-casting entry point against the allocating one.

ntcfd_build_mask_polygon_noalloc serves drivers that rebuild the immersed-
boundary mask inside their time loop (a dynamic angle of attack) or whose
device memory is already handed out, and so cannot call cudaMalloc/cudaFree
there.  It must give exactly the ETA of ntcfd_build_mask_polygon (the masks
are counts, so the test tolerance is zero), call after call, although every
call reuses the same fixed device array.  This file runs last so that a
failure here leaves every other test already run; it also passes alone in a
fresh process, where its first call sets up the array's device address.
"""
import ctypes

import numpy as np
import pytest

from ntustcfdlab_b200 import abi
from ntustcfdlab_b200.abi import dptr, f4, make_params

pytestmark = pytest.mark.gpu


def _solver_and_polygon():
    from ntustcfdlab_b200.solver import Solver, gridder_unequal, naca4_polygon
    n = (3, 96, 120)
    band = (12.5, f4(3.948), f4(3.95), 16, 30, 45, 40, 55, 1.0, f4(0.3), f4(0.6), f4(1.1), 2.0)
    grid = gridder_unequal(*n, 1.0, 8.0, 10.0, band)
    s = Solver(make_params(*n, Re=100.0, dt=1e-3), grid)
    z, y = naca4_polygon(0.12, 256)
    return s, np.ascontiguousarray(z), np.ascontiguousarray(y)


def _noalloc(s, z, y, aoa, zc=4.0, yc=4.0):
    ties = ctypes.c_int(-1)
    rc = s.lib.ntcfd_build_mask_polygon_noalloc(s.h, dptr(z), dptr(y), len(z), aoa, zc, yc,
                                                 ctypes.byref(ties))
    return rc, ties.value


def test_noalloc_mask_matches_allocating_entry_point():
    s, z, y = _solver_and_polygon()
    angles = (5.0, 12.0)
    ref = {}
    for aoa in angles:                      # the allocating entry point
        assert s.build_mask_polygon(z, y, aoa, 4.0, 4.0) == 0
        ref[aoa] = s.get_mask()
    assert not np.array_equal(ref[5.0], ref[12.0])
    s.set_mask(np.zeros(s.halo_shape, order="F"))
    for aoa in angles:                      # two allocation-free calls in a row
        rc, ties = _noalloc(s, z, y, aoa)
        assert rc == 0 and ties == 0, s._err()
        np.testing.assert_array_equal(s.get_mask(), ref[aoa])
    s.close()


def test_noalloc_after_a_larger_call_on_another_context():
    """The shared array still holds a larger plane's flags and list from the
    call before; a smaller context's call must not see them."""
    from ntustcfdlab_b200.solver import Solver, gridder_equal
    s, z, y = _solver_and_polygon()
    assert _noalloc(s, z, y, 7.0) == (0, 0), s._err()
    n = (3, 40, 56)
    s2 = Solver(make_params(*n, Re=100.0, dt=1e-3), gridder_equal(*n, 1.0, 2.0, 2.8))
    try:
        zs, ys = np.ascontiguousarray(z * 0.9), np.ascontiguousarray(y * 0.9)
        assert s2.build_mask_polygon(zs, ys, 9.0, 1.1, 1.0) == 0
        ref = s2.get_mask()
        assert ref.sum() > 0
        s2.set_mask(np.zeros(s2.halo_shape, order="F"))
        for _ in range(2):
            rc, ties = _noalloc(s2, zs, ys, 9.0, 1.1, 1.0)
            assert rc == 0 and ties == 0, s2._err()
            np.testing.assert_array_equal(s2.get_mask(), ref)
    finally:
        s2.close()
        s.close()


def test_noalloc_rejects_inputs_beyond_its_limits():
    s, z, y = _solver_and_polygon()
    big = np.ascontiguousarray(np.resize(z, 16385))
    bigy = np.ascontiguousarray(np.resize(y, 16385))
    rc, _ = _noalloc(s, big, bigy, 5.0)
    assert rc == abi.NTCFD_EINVAL
    assert "at most 16384" in s._err()
    s.close()


def test_noalloc_rejects_a_plane_beyond_its_cell_limit():
    """ny * nz = 513 * 512 > 262144: refused before any device work, with the
    limit in the message; the context stays usable."""
    from ntustcfdlab_b200.solver import Solver, gridder_equal
    n = (3, 513, 512)
    s = Solver(make_params(*n, Re=100.0, dt=1e-3), gridder_equal(*n, 1.0, 4.0, 4.0))
    try:
        z = np.ascontiguousarray([0.5, 1.0, 1.5, 1.0, 0.5])
        y = np.ascontiguousarray([0.0, 0.31, 0.0, -0.29, 0.0])
        rc, _ = _noalloc(s, z, y, 3.0, 1.0, 2.0)
        assert rc == abi.NTCFD_EINVAL
        assert "at most 262144" in s._err()
        assert s.build_mask_polygon(z, y, 3.0, 1.0, 2.0) == 0   # the allocating path takes it
    finally:
        s.close()


def test_noalloc_reports_the_same_ties_as_the_allocating_path():
    """A diamond whose vertices sit on grid nodes: both entry points count the
    same exact vertex/grid ties (the reference would move the grid) and
    refuse the mask; calls after it still work."""
    from ntustcfdlab_b200.solver import Solver, gridder_equal
    n = (3, 32, 32)
    s = Solver(make_params(*n, Re=100.0, dt=1e-3), gridder_equal(*n, 1.0, 4.0, 4.0))
    try:
        z = np.ascontiguousarray([0.5, 1.0, 1.5, 1.0, 0.5])
        y = np.ascontiguousarray([0.0, 0.5, 0.0, -0.5, 0.0])
        ties_ref = ctypes.c_int(-1)
        rc_ref = s.lib.ntcfd_build_mask_polygon(s.h, dptr(z), dptr(y), len(z), 0.0, 1.0, 2.0,
                                                ctypes.byref(ties_ref))
        assert rc_ref == abi.NTCFD_EINVAL and ties_ref.value > 0
        for _ in range(2):
            rc, t = _noalloc(s, z, y, 0.0, 1.0, 2.0)
            assert rc == abi.NTCFD_EINVAL and t == ties_ref.value
            assert "ties" in s._err()
        # a polygon off the nodes (no tie in the oracle either) goes through again:
        # each call clears the shared tie counter
        zo, yo = np.ascontiguousarray(z + 0.0123), np.ascontiguousarray(y + 0.0171)
        rc, t = _noalloc(s, zo, yo, 0.0, 1.0, 2.0)
        assert rc == 0 and t == 0, s._err()
        ref = ctypes.c_int(-1)
        assert s.lib.ntcfd_build_mask_polygon(s.h, dptr(zo), dptr(yo), len(zo), 0.0, 1.0, 2.0,
                                              ctypes.byref(ref)) == 0
        eta = s.get_mask()
        assert _noalloc(s, zo, yo, 0.0, 1.0, 2.0) == (0, 0)
        np.testing.assert_array_equal(s.get_mask(), eta)
    finally:
        s.close()
