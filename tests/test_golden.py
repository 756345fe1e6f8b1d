"""The committed fixtures of tests/golden (made by tests/golden/make_golden.py).

* naca_dat.npz holds a subset of the reference's own airfoil files
  (NACA0012.DAT, NACA0015.DAT, read by airfoil.f90:580-600): the analytic
  polygon generator must reproduce them -- open trailing edge for 0012,
  closed for 0015.
* oracle_*.npz freeze the CPU oracle on small cases; re-running it must give
  the same fields, sweep counts and masks.
"""
import importlib.util
import os

import numpy as np
import pytest

from conftest import interior

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _mg():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _load(name):
    return np.load(os.path.join(GOLD, name))


@pytest.mark.parametrize("name,t,closed", [("naca0012", 0.12, False), ("naca0015", 0.15, True)])
def test_analytic_polygon_reproduces_reference_airfoil_files(ntcfd_lib, name, t, closed):
    from ntustcfdlab_b200.solver import naca4_polygon
    d = _load("naca_dat.npz")[name]
    z, y = naca4_polygon(t, 4096, closed_te=closed)
    up_z, up_y = z[:4096], y[:4096]            # leading edge -> trailing edge, upper surface
    x = np.clip(d[:, 0], 0.0, 1.0)
    dev = np.abs(np.abs(d[:, 1]) - np.interp(x, up_z, up_y))
    body = x < 0.995                           # the files close the trailing edge with extra points
    assert np.median(dev[body]) < 5e-6
    # NACA0012.DAT departs from the polynomial by up to 5e-5 within 3% chord of the nose
    assert dev[body & (x > 0.05)].max() < 2e-5
    # the other trailing-edge choice is clearly worse on the aft body
    z2, y2 = naca4_polygon(t, 4096, closed_te=not closed)
    aft = (x > 0.6) & body
    dev2 = np.abs(np.abs(d[:, 1]) - np.interp(x, z2[:4096], y2[:4096]))
    assert np.median(dev2[aft]) > 10 * np.median(dev[aft])


@pytest.mark.parametrize("tag", ["redblack", "lex"])
def test_oracle_cavity_matches_fixture(orc, tag):
    mg = _mg()
    g = _load(f"oracle_cavity_{tag}.npz")
    f, sweeps = mg.oracle_cavity(mg.SOR_REDBLACK if tag == "redblack" else mg.SOR_LEX)
    assert np.array_equal(sweeps, g["sweeps"])
    for k in "uvwp":
        np.testing.assert_allclose(f[k], g[k], rtol=0, atol=1e-14 * max(1.0, np.abs(g[k]).max()))


def test_oracle_les_cylinder_step_matches_fixture(orc):
    mg = _mg()
    g = _load("oracle_les_cylinder.npz")
    out = mg.oracle_les_step()
    assert np.array_equal(out["ETA"], g["ETA"])
    for k in "uvwp":
        np.testing.assert_allclose(interior(out[k]), interior(g[k]), rtol=0,
                                   atol=1e-13 * np.abs(g[k]).max())
    np.testing.assert_allclose(out["cdrag"], g["cdrag"], rtol=1e-12)
    np.testing.assert_allclose(out["clift"], g["clift"], rtol=1e-12)


def test_oracle_raycasting_of_reference_points_matches_fixture(orc):
    mg = _mg()
    g = _load("oracle_naca0012_dat_mask.npz")
    d = _load("naca_dat.npz")["naca0012"]
    eta, ties = mg.oracle_naca_mask(np.ascontiguousarray(d[:, 0]), np.ascontiguousarray(d[:, 1]))
    assert ties == int(g["ties"][0])
    assert np.array_equal(eta, g["ETA"])


def test_oracle_schemes_reproduce_fixture():
    """The uncalled predictors (discretisation_QUICK/_upwind/_centre.f90)."""
    from oracle import cpu_oracle
    mg = _mg()
    got = mg.oracle_schemes()
    g = _load("oracle_schemes.npz")
    assert sorted(got) == sorted(g.files)
    for k in g.files:
        assert np.array_equal(got[k], g[k]), k
    # the schemes differ from one another
    assert not np.array_equal(g["quick_les_u"], g["centre_les_u"])
    assert not np.array_equal(g["upwind_les_u"], g["centre_les_u"])
