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


def _noalloc(s, z, y, aoa):
    ties = ctypes.c_int(-1)
    rc = s.lib.ntcfd_build_mask_polygon_noalloc(s.h, dptr(z), dptr(y), len(z), aoa, 4.0, 4.0,
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


def test_noalloc_rejects_inputs_beyond_its_limits():
    s, z, y = _solver_and_polygon()
    big = np.ascontiguousarray(np.resize(z, 16385))
    bigy = np.ascontiguousarray(np.resize(y, 16385))
    rc, _ = _noalloc(s, big, bigy, 5.0)
    assert rc == abi.NTCFD_EINVAL
    assert "at most 16384" in s._err()
    s.close()
