"""ctypes mirror of ``include/ntcfd.h`` and the loader of the CUDA library.

The library ``libntcfd.so`` is built in-tree (``ntustcfdlab_b200/lib``) by
``ntustcfdlab_b200.build``.  Loading fails loudly when it is missing: there
is no CPU fallback for the time step.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libntcfd.so")

NTCFD_OK = 0
NTCFD_NOT_CONVERGED = 1
NTCFD_EINVAL = -1
NTCFD_ECUDA = -2
NTCFD_ENOMEM = -3
NTCFD_ENONFINITE = -4
NTCFD_ESTATE = -5
NTCFD_ETIMEOUT = -6

BC_NOSLIP, BC_NEUMANN, BC_DIRICHLET, BC_PERIODIC, BC_INTERFACE = 0, 1, 2, 3, 4
FIELD_U, FIELD_V, FIELD_W, FIELD_P, FIELD_WSTAR, FIELD_E_RED, FIELD_E_BLACK = range(7)
STAGE_PREDICT, STAGE_RHS, STAGE_HALFSWEEP, STAGE_CORRECT, STAGE_PROJECT = range(5)
WEST, EAST, SOUTH, NORTH, BACK, FRONT = 0, 1, 2, 3, 4, 5
FP64, MIXED = 0, 1
QUICK_CENTRE, QUICK, UPWIND, CENTRE = 0, 1, 2, 3   # K2 schemes (discretisation_*.f90)
SMAG_REF_ALIASED, SMAG_STAGGERED = 0, 1
SOR_REDBLACK, SOR_LEX = 0, 1
SOR_AUTO, SOR_STREAMING, SOR_RESIDENT = 0, 1, 2

# boundary-condition strings of variables_module.f90:110-132
BC_NAMES = {"no-slip": BC_NOSLIP, "Neumann": BC_NEUMANN, "Dirichlet": BC_DIRICHLET,
            "periodic": BC_PERIODIC, "interface": BC_INTERFACE}
WALL_NAMES = ("West", "East", "South", "North", "Back", "Front")


class NtcfdParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("Re", ctypes.c_double), ("dt", ctypes.c_double),
        ("omega", ctypes.c_double), ("zeta", ctypes.c_double),
        ("itmax", ctypes.c_int), ("LES", ctypes.c_int),
        ("Cs", ctypes.c_double),
        ("scheme", ctypes.c_int), ("precision", ctypes.c_int),
        ("sor_order", ctypes.c_int), ("smag_mode", ctypes.c_int),
        ("check_every", ctypes.c_int),
        ("bc", (ctypes.c_int * 3) * 6),
        ("bc_value", (ctypes.c_double * 3) * 6),
        ("u_solid", ctypes.c_double * 3),
        ("lx", ctypes.c_double),
        ("mixed_cycle", ctypes.c_int),
        ("diag_divergence", ctypes.c_int),
        ("device", ctypes.c_int),
        ("sor_path", ctypes.c_int),
        ("eager", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
    ]


class NtcfdStepInfo(ctypes.Structure):
    _fields_ = [
        ("sor_iters", ctypes.c_int), ("converged", ctypes.c_int),
        ("sor_last_change", ctypes.c_double),
        ("cDrag", ctypes.c_double), ("cLift", ctypes.c_double),
        ("div_max", ctypes.c_double),
        ("dc_cycles", ctypes.c_int), ("launches", ctypes.c_int),
        ("sor_path", ctypes.c_int), ("pad", ctypes.c_int),
        ("aoa", ctypes.c_double),
    ]


class NtcfdKernelTimes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("predictor_ms", "rhs_ms", "defect_ms", "sweep_ms",
                                              "project_ms", "bc_ms", "resident_ms",
                                              "resident_sweeps")]


class NtcfdAdjSpec(ctypes.Structure):
    _fields_ = [
        ("nsteps", ctypes.c_int), ("checkpoint_every", ctypes.c_int),
        ("w_drag", ctypes.c_double), ("w_lift", ctypes.c_double),
        ("adj_zeta", ctypes.c_double), ("adj_omega", ctypes.c_double), ("adj_itmax", ctypes.c_int),
        ("inflow_wall", ctypes.c_int), ("inflow_normal", ctypes.c_int),
        ("inflow_tangential", ctypes.c_int), ("initial_bc", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
    ]


class NtcfdAdjResult(ctypes.Structure):
    _fields_ = [
        ("J", ctypes.c_double), ("dJ_dbc", (ctypes.c_double * 3) * 6),
        ("dJ_dU", ctypes.c_double), ("dJ_dtheta", ctypes.c_double),
        ("forward_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
        ("recompute_ms", ctypes.c_double), ("solve_ms", ctypes.c_double),
        ("adj_sweeps", ctypes.c_longlong), ("adj_unconverged", ctypes.c_int),
        ("recomputed_steps", ctypes.c_int), ("fwd_status", ctypes.c_int), ("pad", ctypes.c_int),
        ("dJ_daoa_body", ctypes.c_double),
    ]


def f4(x: float) -> float:
    """Value of a Fortran default-real literal stored in a real*8 variable
    (e.g. ``real*8, parameter :: dt = 1.0e-3`` is 0.0010000000474974513)."""
    return float(np.float32(x))


def make_params(nx, ny, nz, *, Re, dt, omega=1.5, zeta=f4(1e-4), itmax=3000, LES=0,
                Cs=f4(0.18), precision=FP64, sor_order=SOR_REDBLACK,
                smag_mode=SMAG_REF_ALIASED, check_every=1, bc=None, bc_value=None,
                u_solid=(0.0, 0.0, 0.0), lx=1.0, mixed_cycle=0,
                diag_divergence=0, device=0, sor_path=SOR_AUTO, eager=0,
                scheme=QUICK_CENTRE) -> NtcfdParams:
    """Builds an ``ntcfd_params``.  ``bc`` maps wall name -> (u, v, w) kind
    strings; missing walls are no-slip, as in variables_module.f90:110-132."""
    p = NtcfdParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.Re, p.dt, p.omega, p.zeta = Re, dt, omega, zeta
    p.itmax, p.LES, p.Cs = itmax, LES, Cs
    p.scheme, p.precision, p.sor_order = scheme, precision, sor_order
    p.smag_mode, p.check_every = smag_mode, check_every
    bc = bc or {}
    bc_value = bc_value or {}
    for wi, wname in enumerate(WALL_NAMES):
        kinds = bc.get(wname, ("no-slip",) * 3)
        vals = bc_value.get(wname, (1.0, 1.0, 1.0))
        for c in range(3):
            p.bc[wi][c] = BC_NAMES[kinds[c]]
            p.bc_value[wi][c] = vals[c]
    for c in range(3):
        p.u_solid[c] = u_solid[c]
    p.lx = lx
    p.mixed_cycle = mixed_cycle
    p.diag_divergence = diag_divergence
    p.device = device
    p.sor_path = sor_path
    p.eager = eager
    return p


def params_copy(p: NtcfdParams, **changes) -> NtcfdParams:
    q = NtcfdParams()
    ctypes.memmove(ctypes.byref(q), ctypes.byref(p), ctypes.sizeof(p))
    for k, v in changes.items():
        setattr(q, k, v)
    return q


_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)

# name -> (restype, argtypes) for every symbol of include/ntcfd.h and
# include/ntcfd_host.h
SIGNATURES = {
    "ntcfd_default_params": (None, [ctypes.POINTER(NtcfdParams)]),
    "ntcfd_create": (ctypes.c_int, [ctypes.POINTER(NtcfdParams), ctypes.POINTER(ctypes.c_void_p)]),
    "ntcfd_destroy": (None, [ctypes.c_void_p]),
    "ntcfd_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "ntcfd_set_metrics": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 6),
    "ntcfd_set_coords": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 3),
    "ntcfd_set_mask": (ctypes.c_int, [ctypes.c_void_p, _DP]),
    "ntcfd_get_mask": (ctypes.c_int, [ctypes.c_void_p, _DP]),
    "ntcfd_build_mask_polygon": (ctypes.c_int, [ctypes.c_void_p, _DP, _DP, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, _IP]),
    "ntcfd_build_mask_polygon_noalloc": (ctypes.c_int, [ctypes.c_void_p, _DP, _DP, ctypes.c_int,
                                                        ctypes.c_double, ctypes.c_double,
                                                        ctypes.c_double, _IP]),
    "ntcfd_build_mask_smooth": (ctypes.c_int, [ctypes.c_void_p, _DP, _DP, ctypes.c_int] + [ctypes.c_double] * 4),
    "ntcfd_build_mask_cylinder": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_double]),
    "ntcfd_set_state": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 4),
    "ntcfd_get_state": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 4),
    "ntcfd_apply_bc": (ctypes.c_int, [ctypes.c_void_p]),
    "ntcfd_get_output": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 4),
    "ntcfd_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                  ctypes.POINTER(NtcfdStepInfo)]),
    "ntcfd_time": (ctypes.c_double, [ctypes.c_void_p]),
    "ntcfd_last_step_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "ntcfd_time_kernels": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                          ctypes.POINTER(NtcfdKernelTimes)]),
    "ntcfd_set_body_force": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 3),
    "ntcfd_set_dynamic_aoa": (ctypes.c_int, [ctypes.c_void_p, _DP, _DP, ctypes.c_int] + [ctypes.c_double] * 4
                              + [ctypes.c_int]),
    "ntcfd_slab_stage": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "ntcfd_slab_change": (ctypes.c_int, [ctypes.c_void_p, _DP]),
    "ntcfd_slab_plane_elems": (ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int]),
    "ntcfd_slab_planes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_int]),
    "ntcfd_output_async": (ctypes.c_int, [ctypes.c_void_p] + [_DP] * 4),
    "ntcfd_output_wait": (ctypes.c_int, [ctypes.c_void_p]),
    "ntcfd_adjoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(NtcfdAdjSpec),
                                     ctypes.POINTER(NtcfdAdjResult), _DP, _DP, _DP,
                                     ctypes.POINTER(NtcfdStepInfo)]),
    # host-side grid generation and geometry (include/ntcfd_host.h)
    "ntcfd_gridder_equal": (None, [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [_DP] * 9),
    "ntcfd_gridder_unequal": (None, [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [_DP] + [_DP] * 9),
    "ntcfd_naca4_polygon": (ctypes.c_int, [ctypes.c_double, ctypes.c_int, _DP, _DP]),
    "ntcfd_naca4_polygon_te": (ctypes.c_int, [ctypes.c_double, ctypes.c_int, ctypes.c_int, _DP, _DP]),
    "ntcfd_circle_polygon": (ctypes.c_int, [ctypes.c_double, ctypes.c_int, _DP, _DP]),
    "ntcfd_write_plot3d_x": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.c_int] * 3 + [_DP] * 3),
    "ntcfd_write_plot3d_q": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.c_int] * 3 + [_DP] * 5 + [ctypes.c_int]),
    "ntcfd_read_plot3d_q": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.c_int] * 3 + [_DP] * 4),
}

_lib = None


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Loads libntcfd.so and binds every declared symbol.  Raises
    FileNotFoundError when the library was not built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m ntustcfdlab_b200.build` "
            "(the time step has no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


def dptr(a: np.ndarray):
    if a.dtype != np.float64 or not (a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]):
        raise TypeError("expected a contiguous float64 array")
    return a.ctypes.data_as(_DP)
