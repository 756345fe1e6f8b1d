"""CPU tests of the product's host side: the C-ABI library loads and exports
every declared symbol, the host grid generators agree with the oracle's
restatement bit for bit, parameter validation happens before any device
call, and the analytic polygons have the reference's ordering."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from ntustcfdlab_b200 import abi
from ntustcfdlab_b200.abi import NtcfdParams, f4, make_params


def _declared_functions():
    names = []
    for hdr in ("ntcfd.h", "ntcfd_host.h"):
        src = open(os.path.join(ROOT, "include", hdr)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(ntcfd_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(ntcfd_lib):
    declared = _declared_functions()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(ntcfd_lib, name), name
        assert name in abi.SIGNATURES, f"{name} has no ctypes signature"


def test_ctypes_struct_layout_matches_header(ntcfd_lib):
    # ntcfd_default_params writes every field; compare with the header defaults
    p = NtcfdParams()
    ntcfd_lib.ntcfd_default_params(ctypes.byref(p))
    assert (p.nx, p.ny, p.nz) == (40, 40, 40)
    assert p.Re == 10.0 and p.dt == f4(1e-3) and p.zeta == f4(1e-4) and p.Cs == f4(0.18)
    assert p.omega == 1.5 and p.itmax == 3000 and p.check_every == 1 and p.lx == 1.0
    assert p.bc[3][2] == abi.BC_DIRICHLET and p.bc[0][0] == abi.BC_NOSLIP
    assert list(p.reserved) == [0] * 3 and p.device == 0 and p.sor_path == abi.SOR_AUTO
    assert p.eager == 0
    # C layout of ntcfd_params on x86-64: 3 ints (+pad), 4 doubles, 2 ints, 1 double,
    # 5 ints, int[6][3], double[6][3], double[3], double, 5 ints, int[3]
    assert ctypes.sizeof(NtcfdParams) == 368


@pytest.mark.parametrize("n", [(7, 9, 11), (40, 40, 40)])
def test_host_gridder_equal_matches_oracle(ntcfd_lib, orc, n):
    from ntustcfdlab_b200.solver import gridder_equal
    a = gridder_equal(*n, 1.0, 2.5, 0.7)
    b = orc.gridder_equal(*n, 1.0, 2.5, 0.7)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_host_gridder_unequal_matches_oracle(ntcfd_lib, orc):
    from ntustcfdlab_b200.solver import gridder_unequal
    band = (f4(12.5), f4(3.948), f4(3.95), 16, 60, 90, 88, 118, 1.0, f4(0.3), f4(0.6), f4(1.1), 2.0)
    a = gridder_unequal(64, 192, 256, 1.0, 8.0, 16.0, band)
    b = orc.gridder_unequal(64, 192, 256, 1.0, 8.0, 16.0, band)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert np.all(a["iDy"] > 0) and np.all(a["iDz"] > 0)


def test_naca_polygon_ordering(ntcfd_lib):
    from ntustcfdlab_b200.solver import naca4_polygon
    z, y = naca4_polygon(0.12, 256)
    assert len(z) == 512
    assert z[0] == 0.0 and y[0] == 0.0 and z[-1] == 0.0 and y[-1] == 0.0     # closed at the LE
    assert np.all(np.diff(z[:256]) > 0) and np.all(y[1:255] > 0)             # upper LE -> TE
    assert np.all(np.diff(z[256:]) < 0) and np.all(y[257:-1] < 0)           # lower TE -> LE
    assert max(y) == pytest.approx(0.06, abs=2e-4)                            # t/2 near x = 0.3


@pytest.mark.parametrize("change,msg", [
    (dict(nx=2), "nx"), (dict(omega=2.0), "omega"), (dict(precision=7), "precision"),
    (dict(sor_order=1), "red-black"), (dict(Re=0.0), "Re"), (dict(itmax=-1), "itmax"),
])
def test_create_rejects_bad_params_before_any_device_call(ntcfd_lib, change, msg):
    p = make_params(8, 8, 8, Re=10.0, dt=1e-3)
    for k, v in change.items():
        setattr(p, k, v)
    h = ctypes.c_void_p()
    rc = ntcfd_lib.ntcfd_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == abi.NTCFD_EINVAL
    assert msg in ntcfd_lib.ntcfd_last_error(h).decode()
    ntcfd_lib.ntcfd_destroy(h)


def test_periodic_must_be_paired(ntcfd_lib):
    p = make_params(8, 8, 8, Re=10.0, dt=1e-3, bc={"West": ("periodic",) * 3})
    h = ctypes.c_void_p()
    assert ntcfd_lib.ntcfd_create(ctypes.byref(p), ctypes.byref(h)) == abi.NTCFD_EINVAL
    assert b"periodic" in ntcfd_lib.ntcfd_last_error(h)
    ntcfd_lib.ntcfd_destroy(h)


def test_product_does_not_import_oracle():
    pat = re.compile(r"(import\s+oracle|from\s+oracle|cpu_oracle|ntcfd_oracle|orc_[a-z])")
    for dp, _, files in os.walk(os.path.join(ROOT, "ntustcfdlab_b200")):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                src = open(os.path.join(dp, f)).read()
                assert not pat.search(src), f
