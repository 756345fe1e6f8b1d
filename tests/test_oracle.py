"""CPU tests of the oracle against closed forms and invariants.

The reference ships no tests or golden vectors and cannot be compiled here
(Fortran + MPI), so the oracle is pinned by the properties below and by the
committed fixtures in tests/golden (generated by tests/golden/make_golden.py).
"""
import numpy as np
import pytest

from conftest import interior, rel_l2
from ntustcfdlab_b200.abi import (SOR_LEX, SOR_REDBLACK, SMAG_STAGGERED, f4, make_params)


def _grid(orc, n=(12, 10, 8), L=(1.0, 1.0, 1.0)):
    return orc.gridder_equal(*n, *L)


def _cavity(orc, n=(12, 10, 8), sor=SOR_REDBLACK, zeta=f4(1e-4), Re=100.0, **kw):
    p = make_params(*n, Re=Re, dt=f4(1e-3), sor_order=sor, zeta=zeta,
                    bc={"North": ("Dirichlet", "no-slip", "no-slip")}, **kw)
    o = orc.Oracle(p, _grid(orc, n))
    o.initial_conditions()
    o.boundary_conditions()
    return o


def test_uniform_metrics_closed_form(orc):
    nx, ny, nz = 10, 7, 5
    g = orc.gridder_equal(nx, ny, nz, 1.0, 2.0, 3.0)
    for key, n, L in (("x", nx, 1.0), ("y", ny, 2.0), ("z", nz, 3.0)):
        X = g[key.upper()]
        iD, Ds = g["iD" + key], g["D" + key + "s"]
        d = L / n
        # X(1) = 0 at index 2, X(-1) = -2d
        assert X[2] == 0.0 and X[0] == -2 * d
        np.testing.assert_allclose(X, (np.arange(n + 5) - 2) * d, rtol=0, atol=1e-13 * L)
        np.testing.assert_allclose(iD, d, rtol=1e-12)
        np.testing.assert_allclose(Ds, d, rtol=1e-12)
        # ghost rules of gridder.f90:121-131
        assert iD[1] == iD[2] and iD[0] == iD[2]
        assert iD[n + 2] == iD[n + 1] and iD[n + 3] == iD[n + 1]
        assert Ds[1] == Ds[2] and Ds[0] == Ds[2]
        assert Ds[n + 1] == Ds[n] and Ds[n + 2] == Ds[n] and Ds[n + 3] == Ds[n]


def test_unequal_grid_bands(orc):
    band = (12.5, 4.0, 4.0, 16, 20, 30, 20, 30, 1.0, 0.4, 0.8, 1.0, 2.0)
    g = orc.gridder_unequal(8, 80, 90, 1.0, 8.0, 12.0, band)
    Y, Z = g["Y"], g["Z"]
    dY = np.diff(Y[2:82])
    assert np.all(dY > 0)
    # three distinct step sizes: small inside the fine band, middle, large
    steps = np.unique(np.round(dY, 9))
    assert len(steps) >= 3
    fine = (Y[2:81] > 3.8) & (Y[2:81] < 4.2)
    # the greedy march uses the fine step inside the fine band (one transition cell aside)
    assert np.median(dY[fine[:len(dY)]]) == pytest.approx(0.4 / 20, rel=1e-9)
    assert np.all(np.diff(Z[2:92]) > 0)


def test_bc_rules_on_small_grid(orc):
    n = (4, 4, 4)
    bc = {"West": ("no-slip", "Neumann", "Dirichlet"), "East": ("Neumann", "no-slip", "no-slip"),
          "North": ("Dirichlet", "no-slip", "no-slip"), "Back": ("no-slip", "Neumann", "no-slip"),
          "Front": ("Neumann", "Neumann", "Neumann")}
    p = make_params(*n, Re=10.0, dt=1e-3, bc=bc)
    o = orc.Oracle(p, _grid(orc, n))
    rng = np.random.default_rng(1)
    fields = {k: rng.standard_normal((8, 8, 8)) for k in "uvwp"}
    for k, a in fields.items():
        o.set(k, a)
    o.boundary_conditions()
    u, v, w, p_ = (o.get(k) for k in "uvwp")
    I = lambda i: i + 1  # Fortran index (from -1) -> array index
    # the last wall written (Front) wins on edges: check interior (j,k) rows of the x walls
    js, ks = slice(I(1), I(4) + 1), slice(I(1), I(4) + 1)
    assert np.all(u[I(0), js, ks] == 0.0) and np.all(u[I(-1), js, ks] == 0.0)
    np.testing.assert_array_equal(v[I(0), js, ks], v[I(1), js, ks])
    np.testing.assert_array_equal(w[I(0), js, ks], 2 * 1.0 - w[I(1), js, ks])
    np.testing.assert_array_equal(u[I(4), js, ks], u[I(3), js, ks])          # East u Neumann
    np.testing.assert_array_equal(u[I(5), js, ks], u[I(4), js, ks])
    np.testing.assert_array_equal(v[I(5), js, ks], -v[I(4), js, ks])
    # lid: u ghost = 2*1 - u(ny)
    is_ = slice(I(1), I(4) + 1)
    np.testing.assert_array_equal(u[is_, I(5), ks], 2.0 - u[is_, I(4), ks])
    assert np.all(v[is_, I(4), ks] == 0.0)
    # BackWall_v Neumann is a no-op on v(i,j,0); v(i,j,-1) copies it
    np.testing.assert_array_equal(v[:, :, I(-1)], v[:, :, I(0)])
    # pressure zero-gradient on every wall
    np.testing.assert_array_equal(p_[I(0), js, ks], p_[I(1), js, ks])
    np.testing.assert_array_equal(p_[is_, is_, I(5)], p_[is_, is_, I(4)])
    # u1 = u2 = u_star = u over the whole halo array
    for k in ("u1", "u2", "u_star"):
        np.testing.assert_array_equal(o.get(k), u)


def test_zero_force_without_body(orc):
    o = _cavity(orc)
    info = o.step(3)
    assert all(i.cDrag == 0.0 and i.cLift == 0.0 for i in info)


def test_projection_reduces_divergence(orc):
    o = _cavity(orc, zeta=1e-13, itmax=20000)
    o.step(2)
    # after the projection with a converged Poisson solve the discrete
    # divergence of u (before the wall values are reset) is at round-off
    o.smagorinsky(); o.predictor()
    o.gauss_seidel()
    o.calcul_new_velocity()
    u2, v2, w2 = o.get("u2"), o.get("v2"), o.get("w2")
    g = o.grid
    iDx, iDy, iDz = g["iDx"][2:-2], g["iDy"][2:-2], g["iDz"][2:-2]
    du = (u2[2:-2, 2:-2, 2:-2] - u2[1:-3, 2:-2, 2:-2]) / iDx[:, None, None]
    dv = (v2[2:-2, 2:-2, 2:-2] - v2[2:-2, 1:-3, 2:-2]) / iDy[None, :, None]
    dw = (w2[2:-2, 2:-2, 2:-2] - w2[2:-2, 2:-2, 1:-3]) / iDz[None, None, :]
    div = du + dv + dw
    us, vs, ws = o.get("u_star"), o.get("v_star"), o.get("w_star")
    dus = (us[2:-2, 2:-2, 2:-2] - us[1:-3, 2:-2, 2:-2]) / iDx[:, None, None]
    dvs = (vs[2:-2, 2:-2, 2:-2] - vs[2:-2, 1:-3, 2:-2]) / iDy[None, :, None]
    dws = (ws[2:-2, 2:-2, 2:-2] - ws[2:-2, 2:-2, 1:-3]) / iDz[None, None, :]
    div_star = dus + dvs + dws
    # frozen pressure ghosts make the walls Dirichlet for p: the flux through
    # the wall faces changes too, so compare away from the walls
    assert np.abs(div[2:-2, 2:-2, 2:-2]).max() < 1e-8 * max(1.0, np.abs(div_star).max())


def test_high_side_wall_faces_are_predicted(orc):
    """discretisation_QUICK_centre.f90 loops i, j, k over 1..n, so u*(nx),
    v*(ny), w*(nz) (the east/north/front wall faces) come from the interior
    formula while u*(0), v*(0), w*(0) keep the boundary values.  The scheme is
    therefore not mirror-symmetric; the wall values come back with the
    end-of-step boundary conditions."""
    n = (10, 10, 10)
    o = _cavity(orc, n)
    o.step(2)
    o.smagorinsky()
    o.predictor()
    ws = o.get("w_star")
    assert np.abs(ws[2:-2, 2:-2, n[2] + 1]).max() > 0.0        # w*(nz) predicted
    assert np.all(ws[:, :, 1] == o.get("w")[:, :, 1])           # w*(0) = w(0) (BC copy)
    o.step(1)
    assert np.all(o.get("w")[2:-2, 2:-2, n[2] + 1] == 0.0)      # no-slip front wall restored


def test_lex_and_redblack_converge_to_same_solution(orc):
    a = _cavity(orc, sor=SOR_LEX, zeta=1e-12, itmax=50000)
    b = _cavity(orc, sor=SOR_REDBLACK, zeta=1e-12, itmax=50000)
    a.step(3)
    b.step(3)
    for k in "uvwp":
        assert rel_l2(interior(a.get(k)), interior(b.get(k))) < 1e-8, k


def test_sor_stop_rule_and_forced_sweeps(orc):
    o = _cavity(orc)
    o.smagorinsky(); o.predictor()
    ik, last, conv = o.gauss_seidel()
    assert conv == 1 and last <= f4(1e-4) and ik >= 1
    o2 = _cavity(orc)
    o2.smagorinsky(); o2.predictor()
    ik2, _, conv2 = o2.gauss_seidel(forced=ik)
    assert ik2 == ik and conv2 == 0
    np.testing.assert_array_equal(o.get("p"), o2.get("p"))


def test_itmax_caps_sweeps(orc):
    o = _cavity(orc, itmax=3, zeta=0.0)
    info = o.step(1)
    assert info[0].sor_iters == 3 and info[0].converged == 0


def test_raycast_square_exact_fractions(orc):
    """A densely sampled axis-aligned square: fully covered cells get 1,
    empty cells 0, cut cells the fraction of 50x50 sub-cell centres inside."""
    nx, ny, nz = 3, 16, 16
    g = orc.gridder_equal(nx, ny, nz, 1.0, 1.0, 1.0)
    p = make_params(nx, ny, nz, Re=10.0, dt=1e-3)
    o = orc.Oracle(p, g)
    z0, z1, y0, y1 = 0.3131, 0.6517, 0.2719, 0.7093
    ns = 64
    t = np.linspace(0, 1, ns, endpoint=False)
    # counter-clockwise, closed: bottom, right, top, left
    zz = np.concatenate([z0 + (z1 - z0) * t, np.full(ns, z1), z1 - (z1 - z0) * t, np.full(ns, z0), [z0]])
    yy = np.concatenate([np.full(ns, y0), y0 + (y1 - y0) * t, np.full(ns, y1), y1 - (y1 - y0) * t, [y0]])
    # RayCasting shifts by the quarter chord and rotates about it; with
    # AoA = 0 and (zc, yc) = (0, 0) the polygon is unchanged
    ties = o.raycasting(zz, yy, 0.0, 0.0, 0.0)
    assert ties == 0
    eta = o.get("ETA")[2, 2:-2, 2:-2]   # i = 1 plane, (j, k)
    h = 1.0 / 16
    for j in range(ny):
        for k in range(nz):
            ya, yb = j * h, (j + 1) * h
            za, zb = k * h, (k + 1) * h
            sy = ya + (np.arange(50) + 0.5) * h / 50
            sz = za + (np.arange(50) + 0.5) * h / 50
            iy = ((sy > y0) & (sy < y1)).sum()
            iz = ((sz > z0) & (sz < z1)).sum()
            expect = iy * iz / 2500.0
            assert eta[j, k] == pytest.approx(expect, abs=1e-12), (j, k)


def test_cylinder_mask_area(orc):
    nx, ny, nz = 4, 48, 48
    g = orc.gridder_equal(nx, ny, nz, 1.0, 6.0, 6.0)
    p = make_params(nx, ny, nz, Re=10.0, dt=1e-3)
    o = orc.Oracle(p, g)
    o.cylinder(3.0, 3.0, 0.5)
    eta = o.get("ETA")[2:-2, 2:-2, 2:-2]
    assert eta.min() >= 0.0 and eta.max() <= 1.0
    assert np.all(eta == eta[:1])                 # extruded along i
    area = eta[0].sum() * (6.0 / 48) ** 2
    assert area == pytest.approx(np.pi * 0.25, rel=2e-3)


def test_force_integral_matches_reference_formula(orc):
    nx, ny, nz = 6, 7, 8
    g = orc.gridder_equal(nx, ny, nz, 1.3, 1.0, 2.0)
    p = make_params(nx, ny, nz, Re=10.0, dt=1e-3, lx=1.3)
    o = orc.Oracle(p, g)
    rng = np.random.default_rng(7)
    FY = np.zeros((nx + 4, ny + 4, nz + 4))
    FZ = np.zeros((nx + 4, ny + 4, nz + 4))
    FY[3:-3, 4:-4, 2:-2] = rng.standard_normal((nx - 2, ny - 4, nz))
    FZ[3:-3, 4:-4, 2:-2] = rng.standard_normal((nx - 2, ny - 4, nz))
    FZ[4, 5, :] = 0.0     # an all-zero column exercises the guard
    o.set("FY", FY)
    o.set("FZ", FZ)
    cd, cl = o.force_integral()
    Dxs, Dys, Dzs = g["Dxs"], g["Dys"], g["Dzs"]
    def integ(F):
        Fz = np.zeros((nx + 2, ny + 2))
        for i in range(1, nx + 1):
            for j in range(1, ny + 1):
                s = 0.0
                for k in range(1, nz + 1):
                    # F(i,j,k) sits at array index (i+1, j+1, k+1), Dzs(k) at k+1
                    s = s + (F[i + 1, j + 1, k] * Dzs[k] + 4.0 * F[i + 1, j + 1, k + 1] * Dzs[k + 1]
                             + F[i + 1, j + 1, k + 2] * Dzs[k + 2]) / 6.0
                Fz[i, j] = s
        Fy = np.zeros(nx + 2)
        for i in range(1, nx + 1):
            s = 0.0
            for j in range(1, ny + 1):
                if Fz[i, j] != 0.0:
                    s = s + (Fz[i, j - 1] * Dys[j] + 4.0 * Fz[i, j] * Dys[j + 1] + Fz[i, j + 1] * Dys[j + 2]) / 6.0
            Fy[i] = s
        t = 0.0
        for i in range(1, nx + 1):
            if Fy[i] != 0.0:
                t = t + (Fy[i - 1] * Dxs[i] + 4.0 * Fy[i] * Dxs[i + 1] + Fy[i + 1] * Dxs[i + 2]) / 6.0
        return t
    assert cd == (-2.0) * integ(FZ) / 1.3
    assert cl == (-2.0) * integ(FY) / 1.3


def test_smagorinsky_modes(orc):
    n = (8, 8, 8)
    p = make_params(*n, Re=100.0, dt=1e-3, LES=1, Cs=f4(0.18))
    o = orc.Oracle(p, _grid(orc, n))
    rng = np.random.default_rng(3)
    for k in "uvw":
        o.set(k, rng.standard_normal((12, 12, 12)))
    o.smagorinsky()
    nut_alias = o.get("Viseff")
    assert np.all(np.isfinite(nut_alias)) and nut_alias.min() >= 0
    p2 = make_params(*n, Re=100.0, dt=1e-3, LES=1, Cs=f4(0.18), smag_mode=SMAG_STAGGERED)
    o2 = orc.Oracle(p2, _grid(orc, n))
    for k in "uvw":
        o2.set(k, o.get(k))
    o2.smagorinsky()
    nut = o2.get("Viseff")
    # the staggered mode with a linear field has the closed-form strain
    x = (np.arange(12) - 2) / 8.0
    lin = np.broadcast_to(x[:, None, None], (12, 12, 12)).copy()
    o2.set("u", lin); o2.set("v", np.zeros((12, 12, 12))); o2.set("w", np.zeros((12, 12, 12)))
    o2.smagorinsky()
    # du/dx = 1 everywhere (two-cell difference over Dxs): |S| term = 2
    delta = (1 / 8.0) ** 3
    expect = (f4(0.18) * delta ** f4(1 / 3)) ** 2 * np.sqrt(2.0)
    np.testing.assert_allclose(o2.get("Viseff"), expect, rtol=1e-6)
    assert not np.allclose(nut, nut_alias)
