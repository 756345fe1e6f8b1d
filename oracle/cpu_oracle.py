"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle
(``oracle/ntcfd_oracle.cpp``).

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this module, as the checker.  The product library never imports it.
Parity status: unpinned by reference tests (the Fortran reference ships none
and cannot be compiled here); the restatement follows the reference file by
file, line by line.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from ntustcfdlab_b200.abi import NtcfdParams, NtcfdStepInfo

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libntcfd_oracle.so")

_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compiles the oracle with its Makefile (g++ -fopenmp); make rebuilds
    when the sources or include/ntcfd.h (the shared structs) changed.  On a
    machine without the compiler the prebuilt library is used as it is."""
    args = ["make", "-C", HERE] + (["-B"] if force else [])
    try:
        subprocess.run(args, check=True, capture_output=True)
    except (FileNotFoundError, subprocess.CalledProcessError):
        if force or not os.path.exists(LIB):
            raise
    return LIB


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        sig = {
            "orc_create": (ctypes.c_void_p, [ctypes.POINTER(NtcfdParams)]),
            "orc_destroy": (None, [ctypes.c_void_p]),
            "orc_set_threads": (None, [ctypes.c_void_p, ctypes.c_int]),
            "orc_set_metrics": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 6),
            "orc_set_coords": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 3),
            "orc_get_coords": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 3),
            "orc_set_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, _DP]),
            "orc_get_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, _DP]),
            "orc_field_size": (ctypes.c_long, [ctypes.c_void_p, ctypes.c_char_p]),
            "orc_initial_conditions": (None, [ctypes.c_void_p]),
            "orc_boundary_conditions": (None, [ctypes.c_void_p]),
            "orc_smagorinsky": (None, [ctypes.c_void_p]),
            "orc_predictor": (None, [ctypes.c_void_p]),
            "orc_gauss_seidel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _DP, _IP]),
            "orc_calcul_new_velocity": (None, [ctypes.c_void_p]),
            "orc_force_integral": (None, [ctypes.c_void_p, _DP, _DP]),
            "orc_updating_velocity": (None, [ctypes.c_void_p]),
            "orc_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                        ctypes.POINTER(NtcfdStepInfo), _IP]),
            "orc_time": (ctypes.c_double, [ctypes.c_void_p]),
            "orc_divergence_max": (ctypes.c_double, [ctypes.c_void_p]),
            "orc_gridder_equal": (None, [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [_DP] * 9),
            "orc_gridder_unequal": (None, [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [_DP] * 10),
            "orc_raycasting": (ctypes.c_int, [ctypes.c_void_p, _DP, _DP, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_double]),
            "orc_cylinder": (None, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64
    return a.ctypes.data_as(_DP)


HALO = {"u", "v", "w", "p", "u1", "v1", "w1", "u2", "v2", "w2", "u_star", "v_star",
        "w_star", "FX", "FY", "FZ", "ETA"}
INNER = {"pre", "uc", "vc", "wc", "Viseff"}


def gridder_equal(nx, ny, nz, lx, ly, lz):
    """Returns dict X, Y, Z, iDx, Dxs, iDy, Dys, iDz, Dzs (gridder.f90:228-327)."""
    X, Y, Z = np.zeros(nx + 5), np.zeros(ny + 5), np.zeros(nz + 5)
    m = [np.zeros(n + 4) for n in (nx, nx, ny, ny, nz, nz)]
    lib().orc_gridder_equal(nx, ny, nz, lx, ly, lz, _p(X), _p(Y), _p(Z), *[_p(a) for a in m])
    return dict(X=X, Y=Y, Z=Z, iDx=m[0], Dxs=m[1], iDy=m[2], Dys=m[3], iDz=m[4], Dzs=m[5])


def gridder_unequal(nx, ny, nz, lx, ly, lz, band):
    """gridder.f90:1-157; band = 13 numbers (see ntcfd_oracle.h)."""
    X, Y, Z = np.zeros(nx + 5), np.zeros(ny + 5), np.zeros(nz + 5)
    m = [np.zeros(n + 4) for n in (nx, nx, ny, ny, nz, nz)]
    b = np.asarray(band, dtype=np.float64)
    lib().orc_gridder_unequal(nx, ny, nz, lx, ly, lz, _p(b), _p(X), _p(Y), _p(Z),
                              *[_p(a) for a in m])
    return dict(X=X, Y=Y, Z=Z, iDx=m[0], Dxs=m[1], iDy=m[2], Dys=m[3], iDz=m[4], Dzs=m[5])


class Oracle:
    """One oracle state (the MODULE variables of variables_module.f90)."""

    def __init__(self, params: NtcfdParams, grid: dict, threads: int = 1):
        self.prm = params
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self.h = lib().orc_create(ctypes.byref(params))
        if not self.h:
            raise ValueError("orc_create rejected the parameters")
        lib().orc_set_threads(self.h, threads)
        self.grid = {k: np.array(v, dtype=np.float64) for k, v in grid.items()}
        g = self.grid
        lib().orc_set_metrics(self.h, _p(g["iDx"]), _p(g["Dxs"]), _p(g["iDy"]), _p(g["Dys"]),
                              _p(g["iDz"]), _p(g["Dzs"]))
        lib().orc_set_coords(self.h, _p(g["X"]), _p(g["Y"]), _p(g["Z"]))

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.orc_destroy(h)
            self.h = None

    # ------------------------------------------------------------ fields
    def shape(self, name):
        if name in HALO:
            return (self.nx + 4, self.ny + 4, self.nz + 4)
        if name in INNER:
            return (self.nx, self.ny, self.nz)
        if name in ("FXz", "FYz"):
            return (self.nx, self.ny)
        return (self.nx,)

    def get(self, name: str) -> np.ndarray:
        a = np.zeros(self.shape(name), dtype=np.float64, order="F")
        if lib().orc_get_field(self.h, name.encode(), _p(a)) != 0:
            raise KeyError(name)
        return a

    def set(self, name: str, a: np.ndarray) -> None:
        a = np.asfortranarray(a, dtype=np.float64)
        if a.shape != self.shape(name):
            raise ValueError(f"{name}: shape {a.shape} != {self.shape(name)}")
        if lib().orc_set_field(self.h, name.encode(), _p(a)) != 0:
            raise KeyError(name)

    def coords(self):
        X, Y, Z = np.zeros(self.nx + 5), np.zeros(self.ny + 5), np.zeros(self.nz + 5)
        lib().orc_get_coords(self.h, _p(X), _p(Y), _p(Z))
        return X, Y, Z

    # ------------------------------------------------------------ stages
    def initial_conditions(self):
        lib().orc_initial_conditions(self.h)

    def boundary_conditions(self):
        lib().orc_boundary_conditions(self.h)

    def smagorinsky(self):
        lib().orc_smagorinsky(self.h)

    def predictor(self):
        lib().orc_predictor(self.h)

    def gauss_seidel(self, forced: int = -1):
        last = ctypes.c_double(0.0)
        conv = ctypes.c_int(0)
        ik = lib().orc_gauss_seidel(self.h, forced, ctypes.byref(last), ctypes.byref(conv))
        return ik, last.value, conv.value

    def calcul_new_velocity(self):
        lib().orc_calcul_new_velocity(self.h)

    def force_integral(self):
        cd, cl = ctypes.c_double(0.0), ctypes.c_double(0.0)
        lib().orc_force_integral(self.h, ctypes.byref(cd), ctypes.byref(cl))
        return cd.value, cl.value

    def updating_velocity(self):
        lib().orc_updating_velocity(self.h)

    def divergence_max(self) -> float:
        return lib().orc_divergence_max(self.h)

    def step(self, nsteps: int = 1, forced=None):
        info = (NtcfdStepInfo * nsteps)()
        fp = None
        if forced is not None:
            f = (ctypes.c_int * nsteps)(*[int(x) for x in forced])
            fp = ctypes.cast(f, _IP)
        lib().orc_step(self.h, nsteps, info, fp)
        return list(info)

    @property
    def time(self) -> float:
        return lib().orc_time(self.h)

    def raycasting(self, az, ay, aoa_deg, zc, yc) -> int:
        az = np.ascontiguousarray(az, dtype=np.float64)
        ay = np.ascontiguousarray(ay, dtype=np.float64)
        return lib().orc_raycasting(self.h, _p(az), _p(ay), len(az), aoa_deg, zc, yc)

    def cylinder(self, zc, yc, r):
        lib().orc_cylinder(self.h, zc, yc, r)
