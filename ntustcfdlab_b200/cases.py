"""Case set-ups: the compile-time configuration of the reference
(variables_module.f90:9-23,56-80,110-132; main.f90:44-70) written out for
the workloads this package is measured on.

Every literal that the reference stores from a default-real constant is
rounded through float32 (``f4``), as the Fortran compiler does for e.g.
``real*8, parameter :: dt = 1.0e-3``.

Axes follow the reference: x is the span (ETA is extruded along i), y the
normal and z the streamwise direction (inflow on the Back wall k = 0,
outflow on the Front wall, boundary_conditions.f90:205-301).
"""
from __future__ import annotations

from dataclasses import dataclass, field

from .abi import FP64, MIXED, SMAG_REF_ALIASED, f4, make_params
from .solver import gridder_equal, gridder_unequal, naca4_polygon


@dataclass
class Case:
    name: str
    params: object
    grid: dict
    steps: int
    mask: dict = field(default_factory=dict)   # {"kind": "naca"|"cylinder", ...}
    description: str = ""

    @property
    def cells(self) -> int:
        return self.params.nx * self.params.ny * self.params.nz


def cavity(n: int, Re: float, dt: float, steps: int, precision=FP64, **kw) -> Case:
    """Lid-driven cavity on the unit cube: no-slip everywhere except the
    y = 1 lid, which moves in x (NorthWall_u = 'Dirichlet', value 1)."""
    p = make_params(n, n, n, Re=Re, dt=f4(dt), precision=precision,
                    bc={"North": ("Dirichlet", "no-slip", "no-slip")}, **kw)
    return Case(name=f"cavity{n}", params=p, grid=gridder_equal(n, n, n, 1.0, 1.0, 1.0),
                steps=steps,
                description=f"lid-driven cavity {n}^3, Re={Re:g}, dt={dt:g}, zero initial fields")


def c1(**kw) -> Case:
    """40^3 cavity, Re=100, dt=1e-3, QUICK, LES off, 200 steps (FP64)."""
    return cavity(40, 100.0, 1e-3, 200, **kw)


def c2(precision=MIXED, **kw) -> Case:
    """128^3 cavity, Re=1000, dt=5e-4, zero initial fields, 500 steps."""
    return cavity(128, 1000.0, 5e-4, 500, precision=precision, **kw)


# Stretched-grid bands for the airfoil cases: the reference's GridderYc/Zc
# and fine-band widths (variables_module.f90:56-80) with cell counts scaled
# to the grid sizes of the cases.
def c3(precision=MIXED, steps: int = 1000, **kw) -> Case:
    """NACA0012 (analytic, 256 cosine points per surface) at AoA 5 deg,
    64 (span x) x 192 (y) x 256 (z) stretched grid over 1 x 8 x 16, body at
    (yc, zc) = (4, 4), Re=1000, inflow w = 1 on the Back wall, Neumann
    outflow, periodic span, Smagorinsky Cs = 0.1, dt = 1e-3."""
    nx, ny, nz = 64, 192, 256
    band = (f4(12.5), f4(3.948), f4(3.95), 16, 60, 90, 88, 118,
            1.0, f4(0.3), f4(0.6), f4(1.1), 2.0)
    grid = gridder_unequal(nx, ny, nz, 1.0, 8.0, 16.0, band)
    bc = {"West": ("periodic",) * 3, "East": ("periodic",) * 3,
          "South": ("Neumann",) * 3, "North": ("Neumann",) * 3,
          "Back": ("Dirichlet", "Dirichlet", "Dirichlet"), "Front": ("Neumann",) * 3}
    bcv = {"Back": (0.0, 0.0, 1.0)}
    p = make_params(nx, ny, nz, Re=1000.0, dt=f4(1e-3), LES=1, Cs=f4(0.1), precision=precision,
                    smag_mode=SMAG_REF_ALIASED, bc=bc, bc_value=bcv, lx=1.0, **kw)
    z, y = naca4_polygon(0.12, 256)
    return Case(name="naca0012_les", params=p, grid=grid, steps=steps,
                mask=dict(kind="naca", az=z, ay=y, aoa=5.0, zc=4.0, yc=4.0),
                description="NACA0012 AoA 5, 64x192x256 stretched, Re 1000, LES Cs 0.1")


def c5(precision=MIXED, steps: int = 2000, **kw) -> Case:
    """NACA0015 (analytic, t = 0.15, closed trailing edge as in the
    reference's NACA0015.DAT, 256 cosine points per surface) at AoA
    10 deg, 128 (span x) x 256 (y) x 384 (z) stretched grid over 1 x 8 x 16
    (12.58 M cells), body at (yc, zc) = (4, 4), Re = 5000, inflow w = 1 on the
    Back wall, Neumann outflow, periodic span, Smagorinsky Cs = 0.1, dt = 5e-4.
    The fine-band cell counts are those of c3 scaled to the larger grid."""
    nx, ny, nz = 128, 256, 384
    band = (f4(12.5), f4(3.948), f4(3.95), 16, 80, 120, 132, 177,
            1.0, f4(0.3), f4(0.6), f4(1.1), 2.0)
    grid = gridder_unequal(nx, ny, nz, 1.0, 8.0, 16.0, band)
    bc = {"West": ("periodic",) * 3, "East": ("periodic",) * 3,
          "South": ("Neumann",) * 3, "North": ("Neumann",) * 3,
          "Back": ("Dirichlet", "Dirichlet", "Dirichlet"), "Front": ("Neumann",) * 3}
    bcv = {"Back": (0.0, 0.0, 1.0)}
    p = make_params(nx, ny, nz, Re=5000.0, dt=f4(5e-4), LES=1, Cs=f4(0.1), precision=precision,
                    smag_mode=SMAG_REF_ALIASED, bc=bc, bc_value=bcv, lx=1.0, **kw)
    z, y = naca4_polygon(0.15, 256, closed_te=True)
    return Case(name="naca0015_les", params=p, grid=grid, steps=steps,
                mask=dict(kind="naca", az=z, ay=y, aoa=10.0, zc=4.0, yc=4.0),
                description="NACA0015 AoA 10, 128x256x384 stretched, Re 5000, LES Cs 0.1")


def cylinder_crossflow(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float, *, zc: float,
                       yc: float, D: float = 1.0, Re: float = 100.0, dt: float = 5e-3, U: float = 1.0,
                       theta_deg: float = 0.0, steps: int = 200, precision=FP64, name="cylinder",
                       **kw) -> Case:
    """Cylinder of diameter D along x (span, periodic) at (zc, yc) on a
    uniform grid; inflow (v, w) = U (sin theta, cos theta) on the Back wall,
    Neumann outflow on the Front wall and Neumann side walls.  ETA comes
    from DFIB_Cylinder (DFIB.f90:74-145)."""
    import math
    bc = {"West": ("periodic",) * 3, "East": ("periodic",) * 3,
          "South": ("Neumann",) * 3, "North": ("Neumann",) * 3,
          "Back": ("Dirichlet", "Dirichlet", "Dirichlet"), "Front": ("Neumann",) * 3}
    th = math.radians(theta_deg)
    bcv = {"Back": (0.0, U * math.sin(th), U * math.cos(th))}
    p = make_params(nx, ny, nz, Re=Re, dt=dt, precision=precision, bc=bc, bc_value=bcv, lx=lx, **kw)
    return Case(name=name, params=p, grid=gridder_equal(nx, ny, nz, lx, ly, lz), steps=steps,
                mask=dict(kind="cylinder", zc=zc, yc=yc, r=0.5 * D),
                description=f"cylinder D={D:g} in cross-flow, {nx}x{ny}x{nz}, Re {Re:g}")


def c4(precision=FP64, **kw) -> Case:
    """Cylinder D = 1, 32 (span x) x 96 (y) x 96 (z) uniform over 4 x 12 x 12,
    centre (zc, yc) = (4, 6), Re = 100, inflow 1, dt = 5e-3; the adjoint runs
    K = 200 steps with a checkpoint every M = 20 steps and a body force
    drawn by body_force_c4()."""
    return cylinder_crossflow(32, 96, 96, 4.0, 12.0, 12.0, zc=4.0, yc=6.0, Re=100.0, dt=f4(5e-3),
                              steps=200, precision=precision, name="cylinder_c4", **kw)


def uniform_inflow_state(case):
    """Impulsive start: the inflow velocity of the Back wall in every cell
    (u = 0, v = U sin theta, w = U cos theta), p = 0, as halo arrays."""
    import numpy as np
    p = case.params
    shape = (p.nx + 4, p.ny + 4, p.nz + 4)
    v0, w0 = p.bc_value[4][1], p.bc_value[4][2]
    z = np.zeros(shape, order="F")
    return (z.copy(), np.full(shape, v0, order="F"), np.full(shape, w0, order="F"), z.copy())


C4_SEED = 20261203


def body_force_c4(shape, seed: int = C4_SEED, scale: float = 1e-3):
    """(fu, fv, fw) ~ N(0, scale) from numpy default_rng(seed), drawn in
    Fortran order one component after the other."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    return tuple(np.reshape(rng.normal(0.0, scale, n), shape, order="F") for _ in range(3))


CASES = {"c1": c1, "c2": c2, "c3": c3, "c4": c4, "c5": c5}
