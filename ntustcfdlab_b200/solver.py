"""Host-side driver of the B200 time step, mirroring the reference's
initialisation and step sequence (main.f90:77-110 then the loop body
main.f90:209-271) over the C-ABI of ``include/ntcfd.h``.

    grid = gridder_equal(nx, ny, nz, lx, ly, lz)       # reading_data + gridder_equal
    s = Solver(params, grid)                           # initial_conditions (all zero)
    s.boundary_conditions()                            # main.f90:100
    s.build_mask_polygon(az, ay, aoa, zc, yc)          # RayCasting, main.f90:109-110
    info = s.step(nsteps)                              # the loop body
    pre, uc, vc, wc = s.get_output()                   # filereachtime fields

Arrays are numpy float64 in Fortran order: halo arrays have shape
(nx+4, ny+4, nz+4), array index i+1 for Fortran index i (-1..n+2).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi
from .abi import NtcfdParams, NtcfdStepInfo, dptr


class NtcfdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ntcfd error {code}: {msg}")
        self.code = code


def _grid_arrays(nx, ny, nz):
    X, Y, Z = np.zeros(nx + 5), np.zeros(ny + 5), np.zeros(nz + 5)
    m = [np.zeros(n + 4) for n in (nx, nx, ny, ny, nz, nz)]
    return X, Y, Z, m


def _grid_dict(X, Y, Z, m):
    return dict(X=X, Y=Y, Z=Z, iDx=m[0], Dxs=m[1], iDy=m[2], Dys=m[3], iDz=m[4], Dzs=m[5])


def gridder_equal(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0) -> dict:
    """reading_data + gridder_equal (reading_data.f90:26-30, gridder.f90:228-327)."""
    lib = abi.load_library()
    X, Y, Z, m = _grid_arrays(nx, ny, nz)
    lib.ntcfd_gridder_equal(nx, ny, nz, lx, ly, lz, dptr(X), dptr(Y), dptr(Z), *[dptr(a) for a in m])
    return _grid_dict(X, Y, Z, m)


def gridder_unequal(nx, ny, nz, lx, ly, lz, band) -> dict:
    """reading_data + gridder_Unequal (reading_data.f90:6-23, gridder.f90:1-157).
    band = (GridderXc, GridderYc, GridderZc, nxSml, nySml, nyMid, nzSml, nzMid,
            lxSml, lySml, lyMid, lzSml, lzMid)."""
    lib = abi.load_library()
    X, Y, Z, m = _grid_arrays(nx, ny, nz)
    b = np.asarray(band, dtype=np.float64)
    lib.ntcfd_gridder_unequal(nx, ny, nz, lx, ly, lz, dptr(b), dptr(X), dptr(Y), dptr(Z),
                              *[dptr(a) for a in m])
    return _grid_dict(X, Y, Z, m)


def naca4_polygon(t: float, npts: int = 256, closed_te: bool = False):
    """Closed analytic NACA 4-digit symmetric section (chord 1), ordered like
    NACA0012.DAT (LE -> upper -> TE -> lower -> LE).  closed_te selects the
    closed trailing-edge coefficient (the form NACA0015.DAT follows)."""
    lib = abi.load_library()
    z, y = np.zeros(2 * npts), np.zeros(2 * npts)
    n = lib.ntcfd_naca4_polygon_te(t, npts, 1 if closed_te else 0, dptr(z), dptr(y))
    return z[:n], y[:n]


def circle_polygon(r: float, npts: int = 128):
    lib = abi.load_library()
    z, y = np.zeros(npts + 1), np.zeros(npts + 1)
    n = lib.ntcfd_circle_polygon(r, npts, dptr(z), dptr(y))
    return z[:n], y[:n]


def write_plot3d_x(path: str, grid: dict):
    """mesh.x of gridder.f90:150-212 (cell-centre coordinates, default reals)."""
    lib = abi.load_library()
    nx, ny, nz = len(grid["X"]) - 5, len(grid["Y"]) - 5, len(grid["Z"]) - 5
    X, Y, Z = (np.ascontiguousarray(grid[k], dtype=np.float64) for k in "XYZ")
    rc = lib.ntcfd_write_plot3d_x(path.encode(), nx, ny, nz, dptr(X), dptr(Y), dptr(Z))
    if rc:
        raise OSError(f"ntcfd_write_plot3d_x({path!r}) returned {rc}")


def write_plot3d_q(path: str, pre, uc, vc, wc, eta, append: bool = True):
    """One NNNN.q solution of filereachtime (filer.f90:161-187): pre, uc, vc, wc
    ((nx, ny, nz)) and the interior of the halo array ETA, appended by default
    as the reference does."""
    lib = abi.load_library()
    nx, ny, nz = pre.shape
    arrs = [np.asfortranarray(a, dtype=np.float64) for a in (pre, uc, vc, wc, eta)]
    rc = lib.ntcfd_write_plot3d_q(path.encode(), nx, ny, nz, *[dptr(a) for a in arrs], 1 if append else 0)
    if rc:
        raise OSError(f"ntcfd_write_plot3d_q({path!r}) returned {rc}")


def read_plot3d_q(path: str, u, v, w, p):
    """reading_variables (reading_data.f90:62-90): fills the halo arrays u, v,
    w, p (Fortran-ordered float64, modified in place) from a .q file."""
    lib = abi.load_library()
    nx, ny, nz = (d - 4 for d in u.shape)
    for a in (u, v, w, p):
        if a.dtype != np.float64 or not a.flags["F_CONTIGUOUS"]:
            raise TypeError("halo arrays must be Fortran-ordered float64")
    rc = lib.ntcfd_read_plot3d_q(path.encode(), nx, ny, nz, dptr(u), dptr(v), dptr(w), dptr(p))
    if rc:
        raise OSError(f"ntcfd_read_plot3d_q({path!r}) returned {rc}")


class Solver:
    """One device-resident grid (an ``ntcfd_ctx``)."""

    def __init__(self, params: NtcfdParams, grid: dict):
        self.lib = abi.load_library()
        self.prm = params
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self._out = None                # arrays of an output_async in flight
        h = ctypes.c_void_p()
        rc = self.lib.ntcfd_create(ctypes.byref(params), ctypes.byref(h))
        self.h = h
        if rc != 0:
            msg = self._err()
            self.close()
            raise NtcfdError(rc, msg)
        self.grid = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in grid.items()}
        g = self.grid
        self._check(self.lib.ntcfd_set_metrics(self.h, dptr(g["iDx"]), dptr(g["Dxs"]), dptr(g["iDy"]),
                                               dptr(g["Dys"]), dptr(g["iDz"]), dptr(g["Dzs"])))
        self._check(self.lib.ntcfd_set_coords(self.h, dptr(g["X"]), dptr(g["Y"]), dptr(g["Z"])))

    # ------------------------------------------------------------ plumbing
    def _err(self) -> str:
        if not self.h:
            return "no context"
        m = self.lib.ntcfd_last_error(self.h)
        return m.decode() if m else ""

    def _check(self, rc: int, allow_warning: bool = False) -> int:
        if rc < 0 or (rc > 0 and not allow_warning):
            raise NtcfdError(rc, self._err())
        return rc

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.ntcfd_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def halo_shape(self):
        return (self.nx + 4, self.ny + 4, self.nz + 4)

    @property
    def inner_shape(self):
        return (self.nx, self.ny, self.nz)

    def _halo(self):
        return np.zeros(self.halo_shape, dtype=np.float64, order="F")

    # ------------------------------------------------------------ state
    def set_state(self, u, v, w, p):
        arrs = [np.asfortranarray(a, dtype=np.float64) for a in (u, v, w, p)]
        for a in arrs:
            if a.shape != self.halo_shape:
                raise ValueError(f"state arrays must have shape {self.halo_shape}")
        self._check(self.lib.ntcfd_set_state(self.h, *[dptr(a) for a in arrs]))

    def get_state(self):
        arrs = [self._halo() for _ in range(4)]
        self._check(self.lib.ntcfd_get_state(self.h, *[dptr(a) for a in arrs]))
        return tuple(arrs)

    def set_mask(self, eta):
        eta = np.asfortranarray(eta, dtype=np.float64)
        self._check(self.lib.ntcfd_set_mask(self.h, dptr(eta)))

    def get_mask(self):
        a = self._halo()
        self._check(self.lib.ntcfd_get_mask(self.h, dptr(a)))
        return a

    def build_mask_polygon(self, az, ay, aoa_deg, zc, yc) -> int:
        """RayCasting (airfoil.f90:580-915) on the device."""
        az = np.ascontiguousarray(az, dtype=np.float64)
        ay = np.ascontiguousarray(ay, dtype=np.float64)
        ties = ctypes.c_int(0)
        self._check(self.lib.ntcfd_build_mask_polygon(self.h, dptr(az), dptr(ay), len(az), aoa_deg,
                                                      zc, yc, ctypes.byref(ties)))
        return ties.value

    def build_mask_smooth(self, az, ay, aoa_deg, zc, yc, width):
        """The body of build_mask_polygon blurred over +-width (a C1 ramp of the
        signed distance); the adjoint then also returns dJ_daoa_body."""
        az = np.ascontiguousarray(az, dtype=np.float64)
        ay = np.ascontiguousarray(ay, dtype=np.float64)
        self._check(self.lib.ntcfd_build_mask_smooth(self.h, dptr(az), dptr(ay), len(az), aoa_deg, zc, yc, width))

    def build_mask_cylinder(self, zc, yc, r):
        """DFIB_Cylinder (DFIB.f90:74-145) on the device."""
        self._check(self.lib.ntcfd_build_mask_cylinder(self.h, zc, yc, r))

    def boundary_conditions(self):
        """boundary_conditions() (boundary_conditions.f90:13-374)."""
        self._check(self.lib.ntcfd_apply_bc(self.h))

    initial_boundary_conditions = boundary_conditions

    def get_output(self):
        """(pre, uc, vc, wc), each (nx, ny, nz) Fortran order."""
        arrs = [np.zeros(self.inner_shape, dtype=np.float64, order="F") for _ in range(4)]
        self._check(self.lib.ntcfd_get_output(self.h, *[dptr(a) for a in arrs]))
        return tuple(arrs)

    def set_dynamic_aoa(self, az, ay, aoa1: float, reduce_frequency: float, zc: float, yc: float,
                        start_step: int):
        """dynamic_AOA + RayCasting before every step from start_step on
        (airfoil.f90:311-321, main.f90:144-155); az=None switches it off."""
        if az is None:
            self._check(self.lib.ntcfd_set_dynamic_aoa(self.h, None, None, 0, 0.0, 0.0, 0.0, 0.0, 0))
            return
        az = np.ascontiguousarray(az, dtype=np.float64)
        ay = np.ascontiguousarray(ay, dtype=np.float64)
        self._check(self.lib.ntcfd_set_dynamic_aoa(self.h, dptr(az), dptr(ay), len(az), aoa1, reduce_frequency,
                                                   zc, yc, start_step))

    def output_async(self, out=None):
        """Start the centred output of the last step without waiting for it.
        `out`: four (nx,ny,nz) Fortran-order float64 arrays to fill (pinned
        ones are written by the copy engine directly), else new ones; they
        are not to be read before output_wait."""
        if out is None:
            out = [np.zeros(self.inner_shape, dtype=np.float64, order="F") for _ in range(4)]
        for a in out:
            assert a.dtype == np.float64 and a.flags.f_contiguous and a.shape == self.inner_shape
        self._check(self.lib.ntcfd_output_async(self.h, *[dptr(a) for a in out]))
        self._out = tuple(out)

    def output_wait(self):
        """(pre, uc, vc, wc) of the last output_async."""
        self._check(self.lib.ntcfd_output_wait(self.h))
        out, self._out = self._out, None
        return out

    def step(self, nsteps: int = 1):
        """Runs the loop body nsteps times; returns (list of NtcfdStepInfo, status).
        status is 0 or NTCFD_NOT_CONVERGED; errors raise."""
        info = (NtcfdStepInfo * max(nsteps, 1))()
        rc = self.lib.ntcfd_step(self.h, nsteps, info)
        self._check(rc, allow_warning=True)
        return list(info)[:nsteps], rc

    @property
    def time(self) -> float:
        return self.lib.ntcfd_time(self.h)

    def last_step_ms(self) -> float:
        """Device time (CUDA events on the context's stream) of the last step() call."""
        ms = ctypes.c_float(0.0)
        self._check(self.lib.ntcfd_last_step_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def time_kernels(self, reps: int = 20) -> dict:
        """Average device time (ms) of standalone launches of the step kernels."""
        t = abi.NtcfdKernelTimes()
        self._check(self.lib.ntcfd_time_kernels(self.h, reps, ctypes.byref(t)))
        return {n: getattr(t, n) for n in ("predictor_ms", "rhs_ms", "defect_ms", "sweep_ms",
                                           "project_ms", "bc_ms", "resident_ms", "resident_sweeps")}

    # ------------------------------------------------------------ adjoint
    def set_body_force(self, fu=None, fv=None, fw=None):
        """Per-cell body force on the u, v, w momentum (each (nx, ny, nz) or None = 0)."""
        arrs = []
        for f in (fu, fv, fw):
            if f is None:
                arrs.append(None)
                continue
            a = np.asfortranarray(f, dtype=np.float64)
            if a.shape != self.inner_shape:
                raise ValueError(f"body force arrays must have shape {self.inner_shape}")
            arrs.append(a)
        ptrs = [dptr(a) if a is not None else None for a in arrs]
        self._check(self.lib.ntcfd_set_body_force(self.h, *ptrs))

    def adjoint(self, nsteps: int, checkpoint_every: int, *, w_drag: float = 1.0,
                w_lift: float = 0.0, adj_zeta: float = 0.0, adj_itmax: int = 0, adj_omega: float = 0.0,
                inflow=None, force_grad: bool = True, initial_bc: bool = False) -> dict:
        """Discrete adjoint of `nsteps` steps from the current state (ntcfd_adjoint).

        J = mean over the steps of (w_drag cDrag + w_lift cLift).  `inflow` =
        (wall, normal component, tangential component) names the Dirichlet
        values that hold U cos(theta), U sin(theta).  initial_bc applies the
        boundary conditions to the state first and differentiates through
        them (otherwise the state, ghosts included, is fixed).  Returns a dict with J,
        dJ_dbc (6x3), dJ_dU, dJ_dtheta, dJ_daoa_body (per radian, with the mask
        of build_mask_smooth), dJ_df (3 arrays or None), the step
        records and the timings; the solver is left after the nsteps steps."""
        spec = abi.NtcfdAdjSpec()
        spec.nsteps, spec.checkpoint_every = nsteps, checkpoint_every
        spec.w_drag, spec.w_lift = w_drag, w_lift
        spec.adj_zeta, spec.adj_itmax, spec.adj_omega = adj_zeta, adj_itmax, adj_omega
        spec.initial_bc = 1 if initial_bc else 0
        if inflow is None:
            spec.inflow_wall, spec.inflow_normal, spec.inflow_tangential = -1, 0, 1
        else:
            wall, cn, ct = inflow
            spec.inflow_wall = abi.WALL_NAMES.index(wall) if isinstance(wall, str) else wall
            spec.inflow_normal, spec.inflow_tangential = cn, ct
        res = abi.NtcfdAdjResult()
        grads = [np.zeros(self.inner_shape, dtype=np.float64, order="F") for _ in range(3)] \
            if force_grad else [None] * 3
        info = (NtcfdStepInfo * nsteps)()
        rc = self.lib.ntcfd_adjoint(self.h, ctypes.byref(spec), ctypes.byref(res),
                                    *[dptr(a) if a is not None else None for a in grads], info)
        self._check(rc, allow_warning=True)
        return {
            "J": res.J,
            "dJ_dbc": np.array([[res.dJ_dbc[w][c] for c in range(3)] for w in range(6)]),
            "dJ_dU": res.dJ_dU, "dJ_dtheta": res.dJ_dtheta, "dJ_daoa_body": res.dJ_daoa_body,
            "dJ_df": grads if force_grad else None,
            "forward_ms": res.forward_ms, "total_ms": res.total_ms,
            "recompute_ms": res.recompute_ms, "solve_ms": res.solve_ms,
            "adj_sweeps": res.adj_sweeps, "adj_unconverged": res.adj_unconverged,
            "recomputed_steps": res.recomputed_steps, "status": rc,
            "info": list(info),
        }
